/*
 * oracle.c - CPU restatement of the reference's hot-path arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product
 * path: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it.  It is never linked into, or called by, the product library.
 *
 * Every function restates one piece of the reference (KHRR-NBody) and cites
 * the file:line it follows.  Operation order matches the reference source
 * (left-to-right sums, no fused multiply-add: build with -ffp-contract=off)
 * so that, compiled the same way, results agree bit-for-bit with the
 * reference's own kernels compiled for the host (oracle/_ref); the tests pin
 * this restatement against fixtures generated from oracle/_ref.
 *
 * Layouts: positions/velocities/accelerations are AoS xyz double triples
 * (the reference's double3), masses and eps^2 are per body.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979 /* common.cuh:7 */
#define ORC_BLOCK 512           /* common.cuh:8 (BLOCK_SIZE) */

/* ------------------------------------------------------------------------ */
/* Analytic halo + bulge field                                               */
/* ------------------------------------------------------------------------ */

/* Field constants: the DataBlock fields dev_fex reads (common.cuh:39-55),
 * derived on the host as nbody/src/nbody.cu:1111-1120 derives them. */
typedef struct {
    double Mh, a, Rh, Mb, b, Rb;
    double Rh2, con, const1, Mh_inf, c_phi_h, c_phi_b;
} orc_field;

void orc_field_init(orc_field* f, double Mh, double a, double Rh, double Mb, double b,
                    double Rb) {
    const double Rh2 = 3.0 * Rh;
    const double rcore1 = Rh / a;
    const double rbcore1 = 1.0 / b;
    const double rbcore2 = rbcore1 * rbcore1;
    const double root1 = sqrt(1.0 + (Rb * Rb) * rbcore2);
    f->Mh = Mh;
    f->a = a;
    f->Rh = Rh;
    f->Mb = Mb;
    f->b = b;
    f->Rb = Rb;
    f->Rh2 = Rh2;
    f->con = Mh / (rcore1 - atan(rcore1));
    f->const1 = Mb / (b * log(Rb * rbcore1 + root1) - Rb / root1);
    f->c_phi_h = f->con / a * (0.5 * log(Rh2 * Rh2 / a / a + 1.0) + atan(Rh2 / a) * a / Rh2) + Mh / Rh2;
    f->c_phi_b = Mb / Rb - f->const1 * log(Rb / b + root1) / Rb;
    f->Mh_inf = Mh * (Rh2 / a - atan(Rh2 / a)) / (rcore1 - atan(rcore1));
}

/* dev_fex (nbody-kernel.cuh:8-40): external acceleration at p. */
static void fex_one(const orc_field* F, const double* p, double* out) {
    const double rr = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    if (rr > 0.0) {
        const double rr3 = rr * rr * rr;
        const double rrcore = rr / F->a;
        const double rrbcore1 = rr / F->b;
        const double root1 = sqrt(1.0 + rrbcore1 * rrbcore1);
        double forcehalo, forceblg1;
        if (rr < F->Rh2) forcehalo = -F->con * (rrcore - atan(rrcore)) / rr3;
        else forcehalo = -F->Mh_inf / rr3;
        if (rr < F->Rb) forceblg1 = -F->const1 * (F->b * log(rrbcore1 + root1) - rr / root1) / rr3;
        else forceblg1 = -F->Mb / rr3;
        const double forcesph = forceblg1 + forcehalo;
        out[0] = forcesph * p[0];
        out[1] = forcesph * p[1];
        out[2] = forcesph * p[2];
    } else {
        out[0] = out[1] = out[2] = 0.0;
    }
}

void orc_fex(const orc_field* F, int64_t n, const double* pos, double* out) {
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) fex_one(F, pos + 3 * i, out + 3 * i);
}

/* ------------------------------------------------------------------------ */
/* Direct sums                                                               */
/* ------------------------------------------------------------------------ */

/* ACCEL_kernel (nbody-kernel.cuh:89-142), FP64: for each target i,
 * a_i = sum_{j=0..n-1} m_j d / (|d|^2 + (eps2_i + eps2_j)/2)^{3/2}, d = r_j - r_i,
 * summed in j order.  out (nt x 3) is overwritten (targets NULL = all). */
void orc_accel_f64(int64_t n, const double* pos, const double* mass, const double* eps2,
                   int64_t nt, const int64_t* targets, double* out) {
    const int64_t count = targets ? nt : n;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t k = 0; k < count; ++k) {
        const int64_t i = targets ? targets[k] : k;
        const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
        const double ei = eps2[i];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            const double dx = pos[3 * j] - xi;
            const double dy = pos[3 * j + 1] - yi;
            const double dz = pos[3 * j + 2] - zi;
            const double den = sqrt(dx * dx + dy * dy + dz * dz + 0.5 * (ei + eps2[j]));
            const double kk = mass[j] / (den * den * den);
            fx += dx * kk;
            fy += dy * kk;
            fz += dz * kk;
        }
        out[3 * k] = fx;
        out[3 * k + 1] = fy;
        out[3 * k + 2] = fz;
    }
}

/* ACCEL_kernel with real = float (the "reference FP32 kernel"): float
 * positions/masses/eps2; the 0.5 literal keeps the softening term in double
 * before the sqrt, whose result is rounded to float (nbody-kernel.cuh:124-131). */
void orc_accel_f32(int64_t n, const double* pos, const double* mass, const double* eps2,
                   int64_t nt, const int64_t* targets, double* out) {
    float* p = (float*)malloc(sizeof(float) * 3 * (size_t)n);
    float* m = (float*)malloc(sizeof(float) * (size_t)n);
    float* e = (float*)malloc(sizeof(float) * (size_t)n);
    for (int64_t i = 0; i < 3 * n; ++i) p[i] = (float)pos[i];
    for (int64_t i = 0; i < n; ++i) {
        m[i] = (float)mass[i];
        e[i] = (float)eps2[i];
    }
    const int64_t count = targets ? nt : n;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t k = 0; k < count; ++k) {
        const int64_t i = targets ? targets[k] : k;
        const float xi = p[3 * i], yi = p[3 * i + 1], zi = p[3 * i + 2];
        const float ei = e[i];
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        for (int64_t j = 0; j < n; ++j) {
            const float dx = p[3 * j] - xi;
            const float dy = p[3 * j + 1] - yi;
            const float dz = p[3 * j + 2] - zi;
            const float d2 = dx * dx + dy * dy + dz * dz;
            const float den = (float)sqrt((double)d2 + 0.5 * (double)(ei + e[j]));
            const float kk = m[j] / (den * den * den);
            fx += dx * kk;
            fy += dy * kk;
            fz += dz * kk;
        }
        out[3 * k] = fx;
        out[3 * k + 1] = fy;
        out[3 * k + 2] = fz;
    }
    free(p);
    free(m);
    free(e);
}

/* PHI_kernel (nbody-kernel.cuh:43-86), FP64: phi_i = -sum_j m_j /
 * sqrt(|d|^2 + (eps2_i + eps2_j)/2), j = i included; out is overwritten. */
void orc_phi_f64(int64_t n, const double* pos, const double* mass, const double* eps2,
                 int64_t nt, const int64_t* targets, double* out) {
    const int64_t count = targets ? nt : n;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t k = 0; k < count; ++k) {
        const int64_t i = targets ? targets[k] : k;
        const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
        const double ei = eps2[i];
        double s = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            const double dx = pos[3 * j] - xi;
            const double dy = pos[3 * j + 1] - yi;
            const double dz = pos[3 * j + 2] - zi;
            s += mass[j] / sqrt(dx * dx + dy * dy + dz * dz + 0.5 * (ei + eps2[j]));
        }
        out[k] = 0.0 - s;
    }
}

/* ------------------------------------------------------------------------ */
/* Predictor-corrector                                                       */
/* ------------------------------------------------------------------------ */

/* kernelNbody_integTime (nbody-kernel.cuh:144-193), one call = one launch.
 * istep 0 (predictor): vel_t = v + dt f, pos_t = r + dt/2 (v + vel_t);
 * istep 1 (corrector): vel_t = (vel_t + v + dt f)/2, pos_t = r, acc0 = acc;
 * f = acc + fex(r).  field NULL means no external field (all constants 0). */
void orc_integ(int64_t n, const orc_field* F, const double* acc, double* pos_t, double* vel_t,
               const double* pos, const double* vel, double dt, int istep, double* acc0) {
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        const double* r = pos + 3 * i;
        const double* v = vel + 3 * i;
        double fe[3] = {0.0, 0.0, 0.0};
        if (F) fex_one(F, r, fe);
        double f[3];
        for (int c = 0; c < 3; ++c) f[c] = acc[3 * i + c] + fe[c];
        if (istep == 0) {
            double vt[3];
            for (int c = 0; c < 3; ++c) vt[c] = v[c] + dt * f[c];
            for (int c = 0; c < 3; ++c) pos_t[3 * i + c] = r[c] + 0.5 * dt * (v[c] + vt[c]);
            for (int c = 0; c < 3; ++c) vel_t[3 * i + c] = vt[c];
        } else {
            double vtt[3];
            for (int c = 0; c < 3; ++c) vtt[c] = 0.5 * (vel_t[3 * i + c] + v[c] + dt * f[c]);
            for (int c = 0; c < 3; ++c) pos_t[3 * i + c] = r[c];
            for (int c = 0; c < 3; ++c) vel_t[3 * i + c] = vtt[c];
            for (int c = 0; c < 3; ++c) acc0[3 * i + c] = acc[3 * i + c];
        }
    }
}

/* The reference time step (nbody/src/nbody.cu:1525-1582): predictor with
 * acc, force at the predicted positions into acct, corrector.  acc (n x 3)
 * carries a(t) in and a(t+dt) out; acct is the force workspace.
 * compat_accumulate != 0 reproduces the reference's missing reset of acct
 * (the force is added onto the previous step's acct); 0 overwrites. */
void orc_run_steps(int64_t n, const orc_field* F, double* pos, double* vel, const double* mass,
                   const double* eps2, double dt, int nsteps, int compat_accumulate, double* acc,
                   double* acct) {
    double* post = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    double* velt = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    double* tmp = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    for (int s = 0; s < nsteps; ++s) {
        orc_integ(n, F, acc, post, velt, pos, vel, dt, 0, acc);
        orc_accel_f64(n, post, mass, eps2, n, NULL, tmp);
        if (compat_accumulate) {
            for (int64_t k = 0; k < 3 * n; ++k) acct[k] += tmp[k];
        } else {
            memcpy(acct, tmp, sizeof(double) * 3 * (size_t)n);
        }
        orc_integ(n, F, acct, pos, vel, post, velt, dt, 1, acc);
    }
    free(post);
    free(velt);
    free(tmp);
}

/* ------------------------------------------------------------------------ */
/* Conservation diagnostics                                                  */
/* ------------------------------------------------------------------------ */

/* result() reductions (nbody/src/nbody.cu:797-833).  out[16] =
 * {Lx, Ly, Lz, Impx, Impy, Impz, Ek, Ep, E, R_max, Z_max, Vr_max, Vfi_max,
 *  Vz_max, 0, 0}; Ek/Ep are the raw sums (E = (Ek + Ep)/2).  Serial order. */
void orc_conservation(int64_t n, const double* pos, const double* vel, const double* mass,
                      const double* psi, double* out) {
    double Lx = 0, Ly = 0, Lz = 0, Ix = 0, Iy = 0, Iz = 0, Ek = 0, Ep = 0;
    double Vr_max = 0, Vfi_max = 0, Vz_max = 0, R_max = 0, Z_max = 0;
    for (int64_t i = 0; i < n; ++i) {
        const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        const double vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2];
        const double r = sqrt(x * x + y * y);
        double vr = 0.0, vfi = 0.0;
        if (r > 0.0) {
            vr = (vx * x + vy * y) / r;
            vfi = (vy * x - vx * y) / r;
        }
        const double m = mass[i];
        Lx += (vz * y - vy * z) * m;
        Ly += (vx * z - vz * x) * m;
        Lz += (vy * x - vx * y) * m;
        Ix += m * vx;
        Iy += m * vy;
        Iz += m * vz;
        Ek += m * (vx * vx + vy * vy + vz * vz);
        Ep += m * psi[i];
        if (fabs(vr) > Vr_max) Vr_max = fabs(vr);
        if (vfi > Vfi_max) Vfi_max = vfi;
        if (fabs(vz) > Vz_max) Vz_max = fabs(vz);
        if (r > R_max) R_max = r;
        if (fabs(z) > Z_max) Z_max = fabs(z);
    }
    out[0] = Lx;
    out[1] = Ly;
    out[2] = Lz;
    out[3] = Ix;
    out[4] = Iy;
    out[5] = Iz;
    out[6] = Ek;
    out[7] = Ep;
    out[8] = 0.5 * (Ek + Ep);
    out[9] = R_max;
    out[10] = Z_max;
    out[11] = Vr_max;
    out[12] = Vfi_max;
    out[13] = Vz_max;
    out[14] = 0.0;
    out[15] = 0.0;
}

/* ------------------------------------------------------------------------ */
/* p2mesh binning                                                            */
/* ------------------------------------------------------------------------ */

/* Cell coordinate of one axis (p2mesh-kernel.cuh:25-36): C truncation toward
 * zero of (p - min)/cs, clamped to [0, g-1].  Out-of-range quotients follow
 * the CUDA float->int conversion (saturating, NaN -> 0), which the clamp then
 * maps to 0 or g-1; inside the int range this is exactly (int) + clamp. */
static int cell_axis(double p, double lo, double cs, int g) {
    const double q = (p - lo) / cs;
    if (q >= (double)(g - 1)) return g - 1;
    if (q > -1.0) return (int)q;
    return 0;
}

/* assignParticlesToCells (p2mesh-kernel.cuh:11-57) in body order, plus the
 * counts.  Note the reference's index quirks, reproduced: iz is clamped to
 * gy-1 and the linear id is iz*gx*gy + iy*gz + ix.
 * cell_id/id_in_cell: n; count: C (zeroed here). */
void orc_assign(int64_t n, const double* pos, const double* lo, const double* cs, const int* g,
                int* cell_id, int* id_in_cell, int* count, int64_t ncells) {
    memset(count, 0, sizeof(int) * (size_t)ncells);
    for (int64_t i = 0; i < n; ++i) {
        const int ix = cell_axis(pos[3 * i], lo[0], cs[0], g[0]);
        const int iy = cell_axis(pos[3 * i + 1], lo[1], cs[1], g[1]);
        const int iz = cell_axis(pos[3 * i + 2], lo[2], cs[2], g[1]);
        const int c = iz * g[0] * g[1] + iy * g[2] + ix;
        cell_id[i] = c;
        id_in_cell[i] = count[c]++;
    }
}

/* Exclusive scan of the counts (the start offsets a correct computePrefixSums
 * would produce), the reference's own start_id view (p2mesh-kernel.cuh:62-123:
 * the in-block scan is discarded, so start_id[c] is the total of all earlier
 * 512-cell blocks), and maxPBC, the inclusive scan of 512-cell block totals
 * that computePrefixSums leaves in its second argument. */
void orc_scan(int64_t ncells, const int* count, int* start_true, int* start_ref, int* maxpbc) {
    const int64_t nb = (ncells + ORC_BLOCK - 1) / ORC_BLOCK;
    int64_t run = 0;
    for (int64_t c = 0; c < ncells; ++c) {
        start_true[c] = (int)run;
        run += count[c];
    }
    int64_t acc = 0;
    for (int64_t b = 0; b < nb; ++b) {
        int64_t tot = 0;
        for (int64_t c = b * ORC_BLOCK; c < (b + 1) * ORC_BLOCK && c < ncells; ++c) tot += count[c];
        const int64_t before = acc;
        acc += tot;
        maxpbc[b] = (int)acc;
        for (int64_t c = b * ORC_BLOCK; c < (b + 1) * ORC_BLOCK && c < ncells; ++c)
            start_ref[c] = (int)before;
    }
}

/* computeCellMassesUnsorted (p2mesh-kernel.cuh:126-137) in body order. */
void orc_cell_masses(int64_t n, const double* mass, const int* cell_id, double* cell_mass,
                     int64_t ncells) {
    memset(cell_mass, 0, sizeof(double) * (size_t)ncells);
    for (int64_t i = 0; i < n; ++i) cell_mass[cell_id[i]] += mass[i];
}

/* computeCellPhiUnsorted (p2mesh-kernel.cuh:152-167) in body order; cell_phi
 * is accumulated into (the reference does not reset it between saves). */
void orc_cell_phi(int64_t n, const double* phi, const int* cell_id, const int* count,
                  double* cell_phi) {
    for (int64_t i = 0; i < n; ++i) cell_phi[cell_id[i]] += phi[i] / count[cell_id[i]];
}

/* ------------------------------------------------------------------------ */
/* Damped-wave Poisson stencil                                               */
/* ------------------------------------------------------------------------ */

typedef struct {
    int nx;
    double dx, dt, c, diss_base, diss_extra, sim_l, bc_l;
} orc_wave;

#define ORC_AT(x, y, z, NX) ((int64_t)(x) + (int64_t)(y) * (NX) + (int64_t)(z) * (NX) * (NX))

/* Sponge coefficient (wave-kernel.cuh:32-60).  Cell coordinates are
 * ix*dx (not centred) and the x test compares against -(L - bc), as the
 * reference does. */
static double wave_diss(const orc_wave* W, int ix, int iy, int iz) {
    const double x = ix * W->dx, y = iy * W->dx, z = iz * W->dx;
    const double L = W->sim_l - W->bc_l;
    double d = W->diss_base;
    if (x > -L) d += W->diss_extra * fabs(x - L) * fabs(x - L);
    else if (x < -L) d += W->diss_extra * fabs(x + L) * fabs(x + L);
    if (y > L) d += W->diss_extra * fabs(y - L) * fabs(y - L);
    else if (y < -L) d += W->diss_extra * fabs(y + L) * fabs(y + L);
    if (z > L) d += W->diss_extra * fabs(z - L) * fabs(z - L);
    else if (z < -L) d += W->diss_extra * fabs(z + L) * fabs(z + L);
    return d;
}

/* wave_diss_iteration (wave-kernel.cuh:5-103), FP64, one full-mesh pass. */
void orc_wave_iter_f64(const orc_wave* W, double* phi_new, const double* phi,
                       const double* phi_old, const double* mass) {
    const int NX = W->nx;
    const double DX = W->dx, C = W->c, DT = W->dt;
#pragma omp parallel for collapse(2)
    for (int iz = 0; iz < NX; ++iz)
        for (int iy = 0; iy < NX; ++iy)
            for (int ix = 0; ix < NX; ++ix) {
                const int64_t at = ORC_AT(ix, iy, iz, NX);
                if (ix == 0 || ix == NX - 1 || iy == 0 || iy == NX - 1 || iz == 0 || iz == NX - 1) {
                    phi_new[at] = 0.0;
                    continue;
                }
                const double rho = mass[at] / (DX * DX * DX);
                const double f = 4 * ORC_PI * 1.0 * rho;
                const double diss = wave_diss(W, ix, iy, iz);
                const double Q = diss * C * DT * 0.5;
                const double Wt = 1 + Q;
                const double K = C * C * (DT * DT) / (DX * DX);
                const double KM = K / Wt;
                const double KF = -(C * C) * (DT * DT) / Wt;
                const double KA = 2 * (1. - 3 * K) / Wt;
                const double KO = (Q - 1.) / Wt;
                phi_new[at] = phi[ORC_AT(ix - 1, iy, iz, NX)] * KM + phi[ORC_AT(ix + 1, iy, iz, NX)] * KM +
                              phi[ORC_AT(ix, iy - 1, iz, NX)] * KM + phi[ORC_AT(ix, iy + 1, iz, NX)] * KM +
                              phi[ORC_AT(ix, iy, iz - 1, NX)] * KM + phi[ORC_AT(ix, iy, iz + 1, NX)] * KM +
                              phi[at] * KA + phi_old[at] * KO + f * KF;
            }
}

/* The product's FP32 form of the same update.  The sponge is separable:
 * diss = base + sx[ix] + sy[iy] + sz[iz], the per-axis terms of wave_diss
 * evaluated in FP64 and rounded once (sz uses the y test, like z does in the
 * reference).  Per interior cell, in FP32: Q = diss c dt/2, w = 1/(1 + Q),
 * out = fma(nb, K w, fma(phi, A w, fma(phi_old, (Q - 1) w, mass (S w))))
 * with nb the six-neighbour sum, K = c^2 dt^2/dx^2, A = 2(1 - 3K),
 * S = -c^2 dt^2 4 pi/dx^3 (constants from FP64).  Algebraically the reference's
 * KM, KA, KO, KF f terms; the FP32 rounding is the product's. */
void orc_wave_iter_f32(const orc_wave* W, float* phi_new, const float* phi, const float* phi_old,
                       const float* mass) {
    const int NX = W->nx;
    const double DX = W->dx, C = W->c, DT = W->dt;
    const double L = W->sim_l - W->bc_l;
    float* sx = (float*)malloc(sizeof(float) * (size_t)NX);
    float* sy = (float*)malloc(sizeof(float) * (size_t)NX);
    for (int i = 0; i < NX; ++i) {
        const double x = i * W->dx;
        double a = 0.0, b = 0.0;
        if (x > -L) a = W->diss_extra * fabs(x - L) * fabs(x - L);
        else if (x < -L) a = W->diss_extra * fabs(x + L) * fabs(x + L);
        if (x > L) b = W->diss_extra * fabs(x - L) * fabs(x - L);
        else if (x < -L) b = W->diss_extra * fabs(x + L) * fabs(x + L);
        sx[i] = (float)a;
        sy[i] = (float)b;
    }
    const double K = C * C * (DT * DT) / (DX * DX);
    const float base = (float)W->diss_base, cdt_half = (float)(C * DT * 0.5), Kf = (float)K;
    const float Af = (float)(2.0 * (1.0 - 3.0 * K));
    const float Sf = (float)(-(C * C) * (DT * DT) * (4.0 * ORC_PI) / (DX * DX * DX));
#pragma omp parallel for collapse(2)
    for (int iz = 0; iz < NX; ++iz)
        for (int iy = 0; iy < NX; ++iy)
            for (int ix = 0; ix < NX; ++ix) {
                const int64_t at = ORC_AT(ix, iy, iz, NX);
                if (ix == 0 || ix == NX - 1 || iy == 0 || iy == NX - 1 || iz == 0 || iz == NX - 1) {
                    phi_new[at] = 0.0f;
                    continue;
                }
                const float nb = ((phi[ORC_AT(ix - 1, iy, iz, NX)] + phi[ORC_AT(ix + 1, iy, iz, NX)]) +
                                  (phi[ORC_AT(ix, iy - 1, iz, NX)] + phi[ORC_AT(ix, iy + 1, iz, NX)])) +
                                 (phi[ORC_AT(ix, iy, iz - 1, NX)] + phi[ORC_AT(ix, iy, iz + 1, NX)]);
                const float diss = ((base + sx[ix]) + sy[iy]) + sy[iz];
                const float Q = diss * cdt_half;
                const float w = 1.0f / (1.0f + Q);
                phi_new[at] = fmaf(nb, Kf * w, fmaf(phi[at], Af * w, fmaf(phi_old[at], (Q - 1.0f) * w, mass[at] * (Sf * w))));
            }
    free(sx);
    free(sy);
}

/* acc_field (p2mesh-kernel.cuh:169-225) over the whole mesh: -grad(phi)/dx
 * by central differences, one-sided on the faces.  cell_acc: C x 3. */
void orc_acc_field(int NX, double DX, const double* phi, double* cell_acc) {
#pragma omp parallel for collapse(2)
    for (int iz = 0; iz < NX; ++iz)
        for (int iy = 0; iy < NX; ++iy)
            for (int ix = 0; ix < NX; ++ix) {
                const int64_t at = ORC_AT(ix, iy, iz, NX);
                double d[3];
                if (ix == 0) d[0] = phi[ORC_AT(ix + 1, iy, iz, NX)] - phi[at];
                else if (ix == NX - 1) d[0] = phi[at] - phi[ORC_AT(ix - 1, iy, iz, NX)];
                else d[0] = 0.5 * (phi[ORC_AT(ix + 1, iy, iz, NX)] - phi[ORC_AT(ix - 1, iy, iz, NX)]);
                if (iy == 0) d[1] = phi[ORC_AT(ix, iy + 1, iz, NX)] - phi[at];
                else if (iy == NX - 1) d[1] = phi[at] - phi[ORC_AT(ix, iy - 1, iz, NX)];
                else d[1] = 0.5 * (phi[ORC_AT(ix, iy + 1, iz, NX)] - phi[ORC_AT(ix, iy - 1, iz, NX)]);
                if (iz == 0) d[2] = phi[ORC_AT(ix, iy, iz + 1, NX)] - phi[at];
                else if (iz == NX - 1) d[2] = phi[at] - phi[ORC_AT(ix, iy, iz - 1, NX)];
                else d[2] = 0.5 * (phi[ORC_AT(ix, iy, iz + 1, NX)] - phi[ORC_AT(ix, iy, iz - 1, NX)]);
                const double coef = -1. / DX;
                cell_acc[3 * at] = d[0] * coef;
                cell_acc[3 * at + 1] = d[1] * coef;
                cell_acc[3 * at + 2] = d[2] * coef;
            }
}

/* apply_acceleration_to_particles + apply_cell_to_particles
 * (p2mesh-kernel.cuh:227-254): NGP gather of cell values to bodies. */
void orc_gather(int64_t n, const int* cell_id, const double* cell_acc, const double* cell_phi,
                double* acc, double* phi) {
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        const int64_t c = cell_id[i];
        if (acc) {
            acc[3 * i] = cell_acc[3 * c];
            acc[3 * i + 1] = cell_acc[3 * c + 1];
            acc[3 * i + 2] = cell_acc[3 * c + 2];
        }
        if (phi) phi[i] = cell_phi[c];
    }
}

/* ------------------------------------------------------------------------ */
/* Beyond the reference's NGP path: cloud-in-cell, the counting sort and the */
/* mesh-force evaluation of its (disabled) Wave mode                         */
/* ------------------------------------------------------------------------ */

/* One CIC axis: u = (p - lo)/cs - 1/2 in cell-centre units, corners floor(u)
 * and floor(u) + 1 with weights 1 - f and f (f = u - floor(u)); coordinates
 * far outside the mesh (and NaN) map to two outside corners.  This is the
 * textbook cloud-in-cell scheme (Hockney & Eastwood, "Computer Simulation
 * Using Particles", ch. 5); the reference deposits NGP only. */
static void cic_axis(double p, double lo, double cs, int g, int* i0, double w[2]) {
    const double u = (p - lo) / cs - 0.5;
    const double fl = floor(u);
    *i0 = fl >= -1.0 ? (fl <= (double)g ? (int)fl : g) : -2;
    const double f = u - fl;
    w[0] = 1.0 - f;
    w[1] = f;
}

/* CIC deposit in body order: cell_mass[c] += m * ((wx * wy) * wz) over the 8
 * corners inside the (cubic) mesh, corners in z, y, x order; cell ids as the
 * binning's (iz*g*g + iy*g + ix). */
void orc_cic_deposit(int64_t n, const double* pos, const double* mass, const double* lo, const double* cs,
                     const int* g, double* cell_mass) {
    for (int64_t i = 0; i < n; ++i) {
        int i0[3];
        double w[3][2];
        for (int k = 0; k < 3; ++k) cic_axis(pos[3 * i + k], lo[k], cs[k], g[k], &i0[k], w[k]);
        for (int c = 0; c < 2; ++c) {
            const int z = i0[2] + c;
            if (z < 0 || z >= g[2]) continue;
            for (int b = 0; b < 2; ++b) {
                const int y = i0[1] + b;
                if (y < 0 || y >= g[1]) continue;
                for (int a = 0; a < 2; ++a) {
                    const int x = i0[0] + a;
                    if (x < 0 || x >= g[0]) continue;
                    const double wt = (w[0][a] * w[1][b]) * w[2][c];
                    cell_mass[(int64_t)z * g[0] * g[1] + (int64_t)y * g[2] + x] += mass[i] * wt;
                }
            }
        }
    }
}

/* CIC interpolation with the same weights: acc = sum w cell_acc, val = sum w
 * cell_val (either output may be NULL), corners in z, y, x order. */
void orc_cic_gather(int64_t n, const double* pos, const double* lo, const double* cs, const int* g,
                    const double* cell_acc, const double* cell_val, double* acc, double* val) {
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        int i0[3];
        double w[3][2];
        for (int k = 0; k < 3; ++k) cic_axis(pos[3 * i + k], lo[k], cs[k], g[k], &i0[k], w[k]);
        double a[3] = {0.0, 0.0, 0.0}, v = 0.0;
        for (int c = 0; c < 2; ++c) {
            const int z = i0[2] + c;
            if (z < 0 || z >= g[2]) continue;
            for (int b = 0; b < 2; ++b) {
                const int y = i0[1] + b;
                if (y < 0 || y >= g[1]) continue;
                for (int x0 = 0; x0 < 2; ++x0) {
                    const int x = i0[0] + x0;
                    if (x < 0 || x >= g[0]) continue;
                    const double wt = (w[0][x0] * w[1][b]) * w[2][c];
                    const int64_t id = (int64_t)z * g[0] * g[1] + (int64_t)y * g[2] + x;
                    if (acc) {
                        a[0] += wt * cell_acc[3 * id];
                        a[1] += wt * cell_acc[3 * id + 1];
                        a[2] += wt * cell_acc[3 * id + 2];
                    }
                    if (val) v += wt * cell_val[id];
                }
            }
        }
        if (acc) {
            acc[3 * i] = a[0];
            acc[3 * i + 1] = a[1];
            acc[3 * i + 2] = a[2];
        }
        if (val) val[i] = v;
    }
}

/* The prefix-sum sort from binning results: order[start[cell_i] + slot_i] = i. */
void orc_scatter_order(int64_t n, const int* cell_id, const int* slot, const int* start, int* order) {
    for (int64_t i = 0; i < n; ++i) order[start[cell_id[i]] + slot[i]] = (int)i;
}

/* One mesh-force evaluation of the reference's Wave mode
 * (calc_acceleration_by_grid, nbody/src/nbody.cu:183-285) on a cubic nx^3
 * mesh over [-nx dx/2, nx dx/2]^3: deposit (cic = 0: the reference's NGP
 * cell of each body, assignParticlesToCells + computeCellMassesUnsorted;
 * cic = 1: the CIC deposit above), `iters` stencil iterations on the ring
 * ring[3] (FP64: ring64, wave_diss_iteration; FP32: ring32, the FP32 form
 * above, masses rounded to float) starting at rotation *rot (old = ring[r],
 * cur = ring[r+1], new -> ring[r+2]), then acc_field on the current field and
 * the gather (NGP: apply_acceleration_to_particles / apply_cell_to_particles;
 * or CIC).  acc (n x 3) and phi (n) receive the body values; *rot advances. */
void orc_mesh_force(const orc_wave* W, int cic, int fp64, int iters, int64_t n, const double* pos,
                    const double* mass, double* ring64, float* ring32, int* rot, double* acc, double* phi) {
    const int NX = W->nx;
    const int64_t C = (int64_t)NX * NX * NX;
    const double L = 0.5 * NX * W->dx;
    const double lo[3] = {-L, -L, -L}, cs[3] = {W->dx, W->dx, W->dx};
    const int g[3] = {NX, NX, NX};
    double* cell_mass = (double*)calloc((size_t)C, sizeof(double));
    int* cell_id = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (cic) {
        orc_cic_deposit(n, pos, mass, lo, cs, g, cell_mass);
    } else {
        for (int64_t i = 0; i < n; ++i) {
            const int ix = cell_axis(pos[3 * i], lo[0], cs[0], g[0]);
            const int iy = cell_axis(pos[3 * i + 1], lo[1], cs[1], g[1]);
            const int iz = cell_axis(pos[3 * i + 2], lo[2], cs[2], g[1]);
            cell_id[i] = iz * g[0] * g[1] + iy * g[2] + ix;
            cell_mass[cell_id[i]] += mass[i];
        }
    }
    double* cur64 = (double*)malloc(sizeof(double) * (size_t)C);
    int r = *rot;
    if (fp64) {
        for (int it = 0; it < iters; ++it, r = (r + 1) % 3)
            orc_wave_iter_f64(W, ring64 + (size_t)((r + 2) % 3) * C, ring64 + (size_t)((r + 1) % 3) * C,
                              ring64 + (size_t)r * C, cell_mass);
        memcpy(cur64, ring64 + (size_t)((r + 1) % 3) * C, sizeof(double) * (size_t)C);
    } else {
        float* m32 = (float*)malloc(sizeof(float) * (size_t)C);
        for (int64_t c = 0; c < C; ++c) m32[c] = (float)cell_mass[c];
        for (int it = 0; it < iters; ++it, r = (r + 1) % 3)
            orc_wave_iter_f32(W, ring32 + (size_t)((r + 2) % 3) * C, ring32 + (size_t)((r + 1) % 3) * C,
                              ring32 + (size_t)r * C, m32);
        const float* cur = ring32 + (size_t)((r + 1) % 3) * C;
        for (int64_t c = 0; c < C; ++c) cur64[c] = (double)cur[c];
        free(m32);
    }
    *rot = r;
    double* cell_acc = (double*)malloc(sizeof(double) * 3 * (size_t)C);
    orc_acc_field(NX, W->dx, cur64, cell_acc);
    if (cic) orc_cic_gather(n, pos, lo, cs, g, cell_acc, cur64, acc, phi);
    else orc_gather(n, cell_id, cell_acc, cur64, acc, phi);
    free(cell_acc);
    free(cur64);
    free(cell_id);
    free(cell_mass);
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
