// GPU time step for the reference channel-dns driver, as a drop-in.
//
// This file defines Simulation::enqueue_serial_step, the single-rank step of
// the reference (src/sim/simulation.cpp:142-171), on top of the cdns C ABI.
// It is meant to be linked into an executable beside the reference's own,
// unmodified sources built as a shared library with -fPIC: the executable's
// definition then takes the place of the library's by ordinary ELF symbol
// interposition (the library calls it through its PLT), so
// Simulation::run (src/sim/simulation.cpp:173-258) and everything around it
// -- config.toml parsing, restart and physical files, statistics,
// diagnostics, disturbance injection -- run exactly as the reference wrote
// them, while the nonlinear term, the RHS assembly, the tau solves and the
// mean-flow correction run on the GPU.  Build recipe and test:
// tests/dropin/Makefile, tests/test_gpu_dropin.py.
//
// State hand-over.  The step keeps the velocity, the multistep history and
// the pressure on the device.  Simulation::run reads the host copies
// (velocity_, pressure_, dpdx_, dpdz_) only after a step whose output branch
// runs (diagnostics, physical, restart or statistics step, the last step) or
// before a disturbance injection; the step computes the same conditions
// (src/sim/simulation.cpp:220-256) and copies the state back exactly then.
// After an injection, which changes velocity_ on the host, the next step
// sends it back with cdns_update_velocity, keeping the history (the
// reference's next step stays second order).  A new run() (its first-order
// first step, recognised by step_coefficients(1)'s a1 = b1 = 0) starts the
// device from the host velocity with cdns_set_velocity.
//
// Errors are thrown as std::runtime_error, as the reference's own step does;
// CDNS_DEVICE selects the CUDA device (default 0).
#include <cstdint>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <string>

#include "cdns.h"
#include "core/mesh.hpp"
#include "core/params.hpp"
#include "sim/initial_bc.hpp"
#include "sim/simulation.hpp"

namespace {

struct DeviceStep {
    cdns_ctx *ctx = nullptr;
    int it = 0;              // Simulation::run's loop counter of the current step
    bool upload = true;      // the host velocity is newer than the device's
    bool restart = true;     // the upload restarts the multistep history
};

// One device context per Simulation object (held until the process exits).
std::map<const Simulation *, DeviceStep> g_steps;

void check(int status, const char *what) {
    if (status == CDNS_OK) return;
    char msg[1024];
    cdns_last_error(msg, sizeof msg);
    throw std::runtime_error(std::string(what) + ": " + msg);
}

double *as_doubles(std::complex<double> *p) { return reinterpret_cast<double *>(p); }
const double *as_doubles(const std::complex<double> *p) { return reinterpret_cast<const double *>(p); }

}  // namespace

void Simulation::enqueue_serial_step(const StepCoefficients &coefficients, double step_time) {
    DeviceStep &g = g_steps[this];
    if (!g.ctx) {
        const cdns_mesh_desc mesh{m_.NX,  m_.NY,  m_.NZ,  m_.NXS,       m_.NYS,       m_.NZS,
                                  m_.NX2, m_.NY2, m_.NZ2, p_.parm.XL, p_.parm.ZL};
        cdns_params params{};
        params.Re = p_.parm.Re;
        params.G_pre = p_.parm.G_pre;
        params.a_pre0 = p_.parm.a_pre0;
        params.b_pre0 = p_.parm.b_pre0;
        for (int k = 0; k < 3; ++k) {
            params.a_V[k] = p_.parm.a_V[k];
            params.b_V[k] = p_.parm.b_V[k];
        }
        params.INDEX_GRAD_PRE = p_.parm.INDEX_GRAD_PRE;
        params.THETA = p_.parm.THETA;
        params.DT = p_.ctrl.DT;
        params.V_Microblow0 = p_.ctrl.V_Microblow0;
        const char *dev = std::getenv("CDNS_DEVICE");
        check(cdns_create(&mesh, &params, CDNS_PRECISION_FP64, dev ? std::atoi(dev) : 0, &g.ctx), "cdns_create");
    }
    // step_coefficients(1) is the only first-order one (src/sim/simulation.cpp:36-45)
    if (coefficients.a1 == 0.0 && coefficients.b1 == 0.0) {
        g.it = 1;
        g.upload = g.restart = true;
    } else {
        ++g.it;
    }
    // the wall data of the step: INDEX_UNSTEADY_BC re-evaluates it at the step's
    // time, as the reference's step body does (src/sim/simulation.cpp:161-164)
    const bool unsteady = p_.parm.INDEX_UNSTEADY_BC == 1;
    if (unsteady) initial_bc::velocity_boundary(velocity_bc_, step_time, p_, m_);
    if (g.upload) {
        if (g.restart)
            check(cdns_set_velocity(g.ctx, as_doubles(velocity_.data())), "cdns_set_velocity");
        else
            check(cdns_update_velocity(g.ctx, as_doubles(velocity_.data())), "cdns_update_velocity");
    }
    if (g.upload || unsteady) check(cdns_set_velocity_bc(g.ctx, as_doubles(velocity_bc_.data())), "cdns_set_velocity_bc");
    g.upload = g.restart = false;
    check(cdns_step(g.ctx, g.it), "cdns_step");

    // Simulation::run's reads of the state after this step (src/sim/simulation.cpp:220-256)
    const std::int64_t ntpit = nt_ + g.it;
    const int physical_interval = p_.physical_interval < 0 ? p_.ctrl.NPRNFRQ : p_.physical_interval;
    const bool diagnostic_step = ntpit % p_.ctrl.NPRNFRQ == 0;
    const bool physical_step = physical_interval > 0 && ntpit % physical_interval == 0;
    const bool restart_step = ntpit % p_.ctrl.NDUMFRQ == 0;
    const bool last_step = g.it == p_.ctrl.NSTEPS;
    const bool sample = ntpit > p_.ctrl.Nstat;
    const bool disturb = disturbances_remaining_ > 0 && ntpit % p_.ctrl.NDISTURBFRQ == 0;
    if (diagnostic_step || physical_step || restart_step || last_step || sample || disturb) {
        check(cdns_synchronize(g.ctx), "time step");
        check(cdns_get_velocity(g.ctx, as_doubles(velocity_.data())), "cdns_get_velocity");
        check(cdns_get_pressure(g.ctx, as_doubles(pressure_.data())), "cdns_get_pressure");
        double dp[2];
        check(cdns_get_dpdx(g.ctx, dp), "cdns_get_dpdx");
        dpdx_ = dp[0];
        dpdz_ = dp[1];
        if (disturb) g.upload = true;   // apply_disturbance changes velocity_ after this step
    }
}
