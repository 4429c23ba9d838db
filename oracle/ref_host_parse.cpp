// oracle/_ref: the reference's galaxy-properties reader, compiled for the host.
//
// TEST INFRASTRUCTURE ONLY.  Wraps read_galaxy_properties and the
// GalaxyProperties accessors (nbody/include/parse.cuh:19-62, 320-367) so the
// tests can compare the product's .ini parser with the reference's own.
#include <cstdio>
#include <filesystem>
#include <format>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "cuda_runtime.h"
#include "parse.cuh"

extern "C" {

// Returns the galaxy count (or -1 when the reader throws).  For each galaxy
// (up to maxg) writes: n_star/n_dark as the accessors report them (a component
// of zero mass has zero bodies), the raw component masses, eps, angle [deg],
// centre xyz and bulk velocity xyz, and the per-body masses.
int ref_read_galaxies(const char* path, int maxg, int* n_star, int* n_dark, double* m_star,
                      double* m_dark, double* eps_star, double* eps_dark, double* angle,
                      double* centre, double* vel, double* m_star_body, double* m_dark_body) {
    try {
        auto g = read_galaxy_properties(std::filesystem::path{path});
        for (int k = 0; k < (int)g.size() && k < maxg; ++k) {
            n_star[k] = g[k].get_n_star_particles();
            n_dark[k] = g[k].get_n_dark_particles();
            m_star[k] = g[k].mass_stars;
            m_dark[k] = g[k].mass_dark;
            eps_star[k] = g[k].eps_stars;
            eps_dark[k] = g[k].eps_dark;
            angle[k] = g[k].angle;
            centre[3 * k + 0] = g[k].pos_center.x;
            centre[3 * k + 1] = g[k].pos_center.y;
            centre[3 * k + 2] = g[k].pos_center.z;
            vel[3 * k + 0] = g[k].vel_center.x;
            vel[3 * k + 1] = g[k].vel_center.y;
            vel[3 * k + 2] = g[k].vel_center.z;
            m_star_body[k] = g[k].get_n_star_particles() ? g[k].get_mass_star_particle() : 0.0;
            m_dark_body[k] = g[k].get_n_dark_particles() ? g[k].get_mass_dark_particle() : 0.0;
        }
        return (int)g.size();
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"
