/*
 * Test harness of the reference-side drop-in (include/shhd_b200_fluid_solver.hpp).
 *
 * Test infrastructure, built by oracle/Makefile (target dropin) from the
 * reference's headers, linked against the CPU checker (oracle/_ref/libshhd_ref.so,
 * which parses the script and builds the reference's Params, Domain2D, models
 * and initial State exactly as Project does) and the engine library.  It
 * constructs B200FluidSolver with FluidSolver's arguments and advances the
 * reference's own State through B200FluidSolver::step(State&, double), so the
 * tests can compare that literal drop-in with the reference's own solver.
 */
#include "ref_harness.h"
#include "shhd_b200_fluid_solver.hpp"

#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>

extern "C" {
void* shref_create(const char* script_text);
void shref_destroy(void* h);
const char* shref_last_error();
}

namespace {

thread_local std::string g_error;

template <typename F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

struct Run {
    void* h = nullptr;
    RefRunView v{};
    explicit Run(const char* script) {
        h = shref_create(script);
        if (!h) throw std::runtime_error(std::string("reference: ") + shref_last_error());
        shref_view(h, v);
    }
    ~Run() { shref_destroy(h); }
};

bool close(double a, double b) { return a == b || std::fabs(a - b) <= 1e-15 * std::max(std::fabs(a), std::fabs(b)); }

}  // namespace

extern "C" {

const char* dropin_last_error() { return g_error.c_str(); }

/* The script's initial state advanced nsteps by B200FluidSolver::step(State&, double), time
 * advancing by dt per step as Project::run_steps does; host_sync 0 every_step, 1 download,
 * 2 resident (then fetch).  out: the State (n doubles). */
int dropin_run(const char* script, int precision, int host_sync, int nsteps, double* out, size_t n) {
    return guarded([&] {
        Run r(script);
        const RefRunView& v = r.v;
        B200FluidSolver solver(*v.params, *v.domain, *v.thermodynamics, *v.free_energy, *v.transport, precision);
        solver.set_host_sync(host_sync == 0 ? B200FluidSolver::HostSync::every_step
                                            : host_sync == 1 ? B200FluidSolver::HostSync::download : B200FluidSolver::HostSync::resident);
        double time = 0.0;
        for (int s = 0; s < nsteps; ++s) {
            solver.step(*v.state, time);
            time += v.params->runtime.dt;
        }
        if (host_sync == 2) solver.fetch(*v.state);
        const size_t have = static_cast<size_t>(v.state->num_fields()) * v.domain->spectral_size() * 2;
        if (n != have) throw std::runtime_error("dropin_run: state size " + std::to_string(have) + " doubles, given " + std::to_string(n));
        std::memcpy(out, v.state->data(), n * sizeof(double));
        return 0;
    });
}

/* 1 when B200FluidSolver's configuration from the reference's Params and model objects equals
 * shhd_config_from_script of the same script in every field the engine reads, else 0 with the
 * first difference in dropin_last_error(). */
int dropin_config_matches(const char* script) {
    return guarded([&] {
        Run r(script);
        const RefRunView& v = r.v;
        const shhd_config a = B200FluidSolver::config_from(*v.params, *v.thermodynamics, *v.free_energy, *v.transport);
        shhd_config b;
        if (shhd_config_from_script(script, &b) != SHHD_OK) throw std::runtime_error(shhd_last_error());
        std::string diff;
        auto cmp = [&](const char* name, double x, double y) {
            if (diff.empty() && !close(x, y)) diff = std::string(name) + ": " + std::to_string(x) + " != " + std::to_string(y);
        };
        cmp("active_nx", a.active_nx, b.active_nx); cmp("active_ny", a.active_ny, b.active_ny);
        cmp("nx", a.nx, b.nx); cmp("ny", a.ny, b.ny); cmp("lx", a.lx, b.lx); cmp("ly", a.ly, b.ly); cmp("dt", a.dt, b.dt);
        cmp("mode", a.mode, b.mode); cmp("integrator", a.integrator, b.integrator);
        cmp("num_order_parameters", a.num_order_parameters, b.num_order_parameters);
        for (int k = 0; k < a.num_order_parameters; ++k) {
            cmp("mu_k0", a.mu_k0[k], b.mu_k0[k]); cmp("mu_k2", a.mu_k2[k], b.mu_k2[k]); cmp("mu_k4", a.mu_k4[k], b.mu_k4[k]);
            // the physical term the engine applies: u psi^3 only under the phi4 style
            cmp("mu_u3", a.free_energy == SHHD_FE_PHI4 ? a.mu_u3[k] : 0.0, b.free_energy == SHHD_FE_PHI4 ? b.mu_u3[k] : 0.0);
            cmp("mobility", a.mobility[k], b.mobility[k]);
        }
        cmp("cT", a.cT, b.cT); cmp("eta", a.eta, b.eta); cmp("zeta", a.zeta, b.zeta);
        cmp("momentum_advection", a.momentum_advection, b.momentum_advection);
        cmp("order_parameter_advection", a.order_parameter_advection, b.order_parameter_advection);
        cmp("noise_momentum", a.noise_momentum, b.noise_momentum);
        cmp("noise_order_parameter", a.noise_order_parameter, b.noise_order_parameter);
        if (a.noise_momentum || a.noise_order_parameter) {
            cmp("noise_seed", static_cast<double>(a.noise_seed), static_cast<double>(b.noise_seed));
            cmp("kBT", a.kBT, b.kBT);
            if (a.noise_order_parameter) cmp("chi", a.chi, b.chi);
        }
        cmp("n_sine_forces", a.n_sine_forces, b.n_sine_forces);
        for (int k = 0; k < a.n_sine_forces; ++k) {
            cmp("sine.target", a.sine_forces[k].target, b.sine_forces[k].target);
            cmp("sine.component", a.sine_forces[k].component, b.sine_forces[k].component);
            cmp("sine.axis", a.sine_forces[k].axis, b.sine_forces[k].axis);
            cmp("sine.nk", a.sine_forces[k].nk, b.sine_forces[k].nk);
            cmp("sine.amplitude", a.sine_forces[k].amplitude, b.sine_forces[k].amplitude);
        }
        cmp("n_gradient_forces", a.n_gradient_forces, b.n_gradient_forces);
        for (int k = 0; k < a.n_gradient_forces; ++k) {
            cmp("gradient.component", a.gradient_forces[k].component, b.gradient_forces[k].component);
            cmp("gradient.direction", a.gradient_forces[k].direction, b.gradient_forces[k].direction);
            cmp("gradient.amplitude", a.gradient_forces[k].amplitude, b.gradient_forces[k].amplitude);
        }
        if (!diff.empty()) {
            g_error = diff;
            return 0;
        }
        return 1;
    });
}

}  // extern "C"
