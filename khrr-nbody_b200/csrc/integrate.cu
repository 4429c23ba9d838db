// FP64 predictor-corrector, external field and conservation sums on sm_100a.
//
// Replaces kernelNbody_integTime (nbody-kernel.cuh:144-193) with dev_fex
// (nbody-kernel.cuh:8-40), the reference's step sequencing
// (nbody/src/nbody.cu:1525-1582) and the host FP64 loop of result()
// (nbody/src/nbody.cu:797-833).  All of it is HBM-bound FP64 work.
//
// The time step is  predictor -> force -> corrector.  Because the corrector
// leaves x(t+dt) = x* and the next predictor only needs x(t+dt), v(t+dt) and
// a(t+dt) (plus fex at the same x), the corrector of step k and the predictor
// of step k+1 are fused into one pass ("kick-drift"), which also writes the
// FP32 shadow (x*, m) the next force pass reads.  The arithmetic is the
// reference's, operation for operation; this file is built with FMA
// contraction off so the results equal the reference's expressions evaluated
// in IEEE double.
#include <cmath>
#include <cstdint>

#include "khrr_internal.h"

namespace khrr {

FieldConsts make_field(double Mh, double a, double Rh, double Mb, double b, double Rb) {
    // Host constants as nbody/src/nbody.cu:1111-1120 derives them.
    FieldConsts f{};
    const double Rh2 = 3.0 * Rh;
    const double rcore1 = Rh / a;
    const double rbcore1 = 1.0 / b;
    const double rbcore2 = rbcore1 * rbcore1;
    const double root1 = std::sqrt(1.0 + (Rb * Rb) * rbcore2);
    f.a = a;
    f.b = b;
    f.Rb = Rb;
    f.Mb = Mb;
    f.Rh2 = Rh2;
    f.con = Mh / (rcore1 - std::atan(rcore1));
    f.const1 = Mb / (b * std::log(Rb * rbcore1 + root1) - Rb / root1);
    f.Mh_inf = Mh * (Rh2 / a - std::atan(Rh2 / a)) / (rcore1 - std::atan(rcore1));
    f.enabled = 1;
    return f;
}

namespace {

struct d3 {
    double x, y, z;
};

__device__ __forceinline__ d3 ld3(const double* p, int64_t i) {
    return d3{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
}

__device__ __forceinline__ void st3(double* p, int64_t i, const d3& v) {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}

// dev_fex (nbody-kernel.cuh:8-40): static halo + bulge acceleration at p.
__device__ d3 fex(const FieldConsts& F, const d3& p) {
    if (!F.enabled) return d3{0.0, 0.0, 0.0};
    const double rr = sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
    if (!(rr > 0.0)) return d3{0.0, 0.0, 0.0};
    const double rr3 = rr * rr * rr;
    const double rrcore = rr / F.a;
    const double rrbcore1 = rr / F.b;
    const double root1 = sqrt(1.0 + rrbcore1 * rrbcore1);
    const double forcehalo = rr < F.Rh2 ? -F.con * (rrcore - atan(rrcore)) / rr3 : -F.Mh_inf / rr3;
    const double forceblg1 =
        rr < F.Rb ? -F.const1 * (F.b * log(rrbcore1 + root1) - rr / root1) / rr3 : -F.Mb / rr3;
    const double s = forceblg1 + forcehalo;
    return d3{s * p.x, s * p.y, s * p.z};
}

// Positions of the FP32 shadow (its masses and softenings never change).
__device__ __forceinline__ void write_shadow(const Shadow& sh, int64_t i, const d3& p) {
    sh.x[i] = static_cast<float>(p.x);
    sh.y[i] = static_cast<float>(p.y);
    sh.z[i] = static_cast<float>(p.z);
}

// Predictor (istep 0): v* = v + dt f, x* = x + dt/2 (v + v*), f = a + fex(x).
__device__ __forceinline__ void predict(const StepArgs& a, int64_t i, const d3& r, const d3& v,
                                        const d3& f) {
    d3 vt, pt;
    vt.x = v.x + a.dt * f.x;
    vt.y = v.y + a.dt * f.y;
    vt.z = v.z + a.dt * f.z;
    pt.x = r.x + 0.5 * a.dt * (v.x + vt.x);
    pt.y = r.y + 0.5 * a.dt * (v.y + vt.y);
    pt.z = r.z + 0.5 * a.dt * (v.z + vt.z);
    st3(a.post, i, pt);
    st3(a.velt, i, vt);
    write_shadow(a.shadow, i, pt);
}

__global__ void predictor_kernel(const StepArgs a) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const d3 r = ld3(a.pos, i), v = ld3(a.vel, i), ac = ld3(a.acc, i);
        const d3 fe = fex(a.field, r);
        const d3 f{ac.x + fe.x, ac.y + fe.y, ac.z + fe.z};
        predict(a, i, r, v, f);
    }
}

__device__ __forceinline__ void sum_partials(const StepArgs& a, int64_t i, d3& s, double& sp) {
    s = d3{0.0, 0.0, 0.0};
    sp = 0.0;
    if (a.fx) {
        // The pair kernel's fixed-point sums (zero for ghosts).
        const FxScale sc = a.fx_scale[i / kPad];
        s.x = static_cast<double>(static_cast<long long>(a.fx[i])) * sc.inv_acc;
        s.y = static_cast<double>(static_cast<long long>(a.fx[a.npad + i])) * sc.inv_acc;
        s.z = static_cast<double>(static_cast<long long>(a.fx[2 * a.npad + i])) * sc.inv_acc;
        sp = static_cast<double>(static_cast<long long>(a.fx[3 * a.npad + i])) * sc.inv_phi;
        return;
    }
    const int ns = a.nsplit[i];
    for (int k = 0; k < ns; ++k) {
        const double4 p = a.part[k * a.npad + i];
        s.x += p.x;
        s.y += p.y;
        s.z += p.z;
        sp += p.w;
    }
}

// Corrector (istep 1) fused with the next predictor.
__global__ void corrector_kernel(const StepArgs a) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        d3 an;
        double sp;
        sum_partials(a, i, an, sp);
        if (a.compat_accumulate) {
            // The reference adds each step's force onto acct_ (never zeroed).
            d3 prev = ld3(a.acct, i);
            an = d3{prev.x + an.x, prev.y + an.y, prev.z + an.z};
            st3(a.acct, i, an);
        }
        const d3 xs = ld3(a.post, i), vs = ld3(a.velt, i), vo = ld3(a.vel, i);
        const d3 fe = fex(a.field, xs);
        const d3 f{an.x + fe.x, an.y + fe.y, an.z + fe.z};
        d3 vn;
        vn.x = 0.5 * (vo.x + vs.x + a.dt * f.x);
        vn.y = 0.5 * (vo.y + vs.y + a.dt * f.y);
        vn.z = 0.5 * (vo.z + vs.z + a.dt * f.z);
        st3(a.pos, i, xs);
        st3(a.vel, i, vn);
        st3(a.acc, i, an);
        if (a.want_phi) a.phi[i] = 0.0 - sp;
        if (a.predict_next) predict(a, i, xs, vn, f);
    }
}

// Partials -> state acc/phi (khrr_forces).
__global__ void collect_kernel(const StepArgs a, int want_acc, int accumulate) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        d3 s;
        double sp;
        sum_partials(a, i, s, sp);
        if (want_acc) {
            if (accumulate) {
                const d3 prev = ld3(a.acc, i);
                s = d3{prev.x + s.x, prev.y + s.y, prev.z + s.z};
            }
            st3(a.acc, i, s);
        }
        if (a.want_phi) a.phi[i] = 0.0 - sp;
    }
}

// kernelNbody_integTime (nbody-kernel.cuh:144-193) with its argument roles.
__global__ void integ_time_kernel(const double* acc, double* pos_t, double* vel_t, const double* pos,
                                  const double* vel, double dt, int istep, double* acc0, int64_t n,
                                  const FieldConsts F) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const d3 v = ld3(vel, i), r = ld3(pos, i), ac = ld3(acc, i);
        const d3 fe = fex(F, r);
        const d3 f{ac.x + fe.x, ac.y + fe.y, ac.z + fe.z};
        if (istep == 0) {
            d3 vt, pt;
            vt.x = v.x + dt * f.x;
            vt.y = v.y + dt * f.y;
            vt.z = v.z + dt * f.z;
            pt.x = r.x + 0.5 * dt * (v.x + vt.x);
            pt.y = r.y + 0.5 * dt * (v.y + vt.y);
            pt.z = r.z + 0.5 * dt * (v.z + vt.z);
            st3(pos_t, i, pt);
            st3(vel_t, i, vt);
        } else {
            const d3 vt = ld3(vel_t, i);
            d3 vtt;
            vtt.x = 0.5 * (vt.x + v.x + dt * f.x);
            vtt.y = 0.5 * (vt.y + v.y + dt * f.y);
            vtt.z = 0.5 * (vt.z + v.z + dt * f.z);
            st3(pos_t, i, r);
            st3(vel_t, i, vtt);
            st3(acc0, i, ac);
        }
    }
}

// ---- conservation sums (result(), nbody/src/nbody.cu:797-833) ---------------
// 8 sums (Lx Ly Lz Ix Iy Iz Ek Ep) + 5 maxima (R Z |Vr| Vfi |Vz|) per block,
// then one block folds the block results in index order: deterministic.
constexpr int kConsThreads = 256;
constexpr int kConsFields = 13;

__global__ void conservation_blocks_kernel(const double* pos, const double* vel, const double* mass,
                                           const double* phi, int64_t n, double* block_out) {
    double v[kConsFields];
#pragma unroll
    for (int k = 0; k < kConsFields; ++k) v[k] = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        const double vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2];
        const double m = mass[i];
        const double r = sqrt(x * x + y * y);
        double vr = 0.0, vfi = 0.0;
        if (r > 0.0) {
            vr = (vx * x + vy * y) / r;
            vfi = (vy * x - vx * y) / r;
        }
        v[0] += (vz * y - vy * z) * m;
        v[1] += (vx * z - vz * x) * m;
        v[2] += (vy * x - vx * y) * m;
        v[3] += m * vx;
        v[4] += m * vy;
        v[5] += m * vz;
        v[6] += m * (vx * vx + vy * vy + vz * vz);
        v[7] += m * phi[i];
        v[8] = fmax(v[8], r);
        v[9] = fmax(v[9], fabs(z));
        v[10] = fmax(v[10], fabs(vr));
        v[11] = fmax(v[11], vfi);
        v[12] = fmax(v[12], fabs(vz));
    }
    __shared__ double sh[kConsFields][kConsThreads];
#pragma unroll
    for (int k = 0; k < kConsFields; ++k) sh[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int w = kConsThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
#pragma unroll
            for (int k = 0; k < 8; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
#pragma unroll
            for (int k = 8; k < kConsFields; ++k)
                sh[k][threadIdx.x] = fmax(sh[k][threadIdx.x], sh[k][threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x < kConsFields) block_out[blockIdx.x * kConsFields + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void conservation_final_kernel(const double* block_out, int nblocks, double* out16) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double v[kConsFields];
    for (int k = 0; k < kConsFields; ++k) v[k] = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        for (int k = 0; k < 8; ++k) v[k] += block_out[b * kConsFields + k];
        for (int k = 8; k < kConsFields; ++k) v[k] = fmax(v[k], block_out[b * kConsFields + k]);
    }
    // Layout of khrr_lie: L[3], Imp[3], Ek, Ep, E, R_max, Z_max, Vr_max, Vfi_max, Vz_max.
    for (int k = 0; k < 8; ++k) out16[k] = v[k];
    out16[8] = 0.5 * (v[6] + v[7]);
    out16[9] = v[8];
    out16[10] = v[9];
    out16[11] = v[10];
    out16[12] = v[11];
    out16[13] = v[12];
    out16[14] = 0.0;
    out16[15] = 0.0;
}

int grid_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    if (g > 148 * 16) g = 148 * 16;
    if (g < 1) g = 1;
    return static_cast<int>(g);
}

}  // namespace

cudaError_t launch_predictor(const StepArgs& a, cudaStream_t s) {
    predictor_kernel<<<grid_for(a.n, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_corrector(const StepArgs& a, cudaStream_t s) {
    corrector_kernel<<<grid_for(a.n, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_collect(const StepArgs& a, bool want_acc, bool accumulate, cudaStream_t s) {
    collect_kernel<<<grid_for(a.n, 256), 256, 0, s>>>(a, want_acc ? 1 : 0, accumulate ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_integ_time(const double* acc, double* pos_t, double* vel_t, const double* pos,
                              const double* vel, double dt, int istep, double* acc0, int64_t n,
                              const FieldConsts& f, cudaStream_t s) {
    integ_time_kernel<<<grid_for(n, 256), 256, 0, s>>>(acc, pos_t, vel_t, pos, vel, dt, istep, acc0,
                                                       n, f);
    return cudaGetLastError();
}

int conservation_blocks(int64_t n) {
    int64_t b = (n + kConsThreads - 1) / kConsThreads;
    if (b > 148 * 4) b = 148 * 4;
    if (b < 1) b = 1;
    return static_cast<int>(b);
}

cudaError_t launch_conservation(const double* pos, const double* vel, const double* mass,
                                const double* phi, int64_t n, double* block_out, int nblocks,
                                double* out16, cudaStream_t s) {
    conservation_blocks_kernel<<<nblocks, kConsThreads, 0, s>>>(pos, vel, mass, phi, n, block_out);
    conservation_final_kernel<<<1, 32, 0, s>>>(block_out, nblocks, out16);
    return cudaGetLastError();
}

}  // namespace khrr
