/*
 * C-ABI harness around the reference solver's own classes (oracle only).
 *
 * Test infrastructure: built by oracle/Makefile together with the
 * reference's unmodified src .cc files into oracle/_ref/libshhd_ref.so, against
 * the single-rank shims in oracle/ref_shim/.  It is the CPU checker and the
 * timed CPU baseline; nothing in the product links it.
 *
 * It repeats what Project does (src/project.h:92-145): parse the input
 * script with ParamParser, build Domain2D / SpectralMask2D / State, create
 * the models through the registries (project.h:59-90), apply the initial
 * conditions (project.h:92-116), then advance with the same
 * FCalculator + TimeIntegrator pair FluidSolver wires (fluid_solver.h:37-99).
 * The one addition is that the RHSOperators it binds copy each psi_sto /
 * j_sto output aside, so the noise the reference drew can be replayed.
 * The script's `measure` commands run through the reference's own
 * MeasurementManager after every step of shref_step, with the integrator's
 * flux buffer, as Project::run_steps does (project.h:127-143);
 * shref_finalize closes their files.
 */
#include "ref_harness.h"

#include "domain.h"
#include "fcalculator.h"
#include "fcalculator_dynamics_mode.h"
#include "initial_condition.h"
#include "fourier_transform.h"
#include "initial_condition_registry_builtin.h"
#include "measure_manager.h"
#include "measure_registry_builtin.h"
#include "model_free_energy_null.h"
#include "model_free_energy_registry_builtin.h"
#include "model_thermodynamics_null.h"
#include "model_thermodynamics_registry_builtin.h"
#include "model_transport_coefficient_registry_builtin.h"
#include "param_parser.h"
#include "simulationinfo.h"
#include "spectral_mask.h"
#include "state.h"
#include "time_integrator.h"
#include "time_integrator_euler_compressible.h"
#include "time_integrator_euler_incompressible.h"
#include "time_integrator_euler_quiescent.h"
#include "time_integrator_srk3_compressible.h"
#include "time_integrator_srk3_incompressible.h"
#include "time_integrator_srk3_quiescent.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <unistd.h>
#include <vector>

namespace {

thread_local std::string g_error;

struct RefRun {
    Params params;
    std::unique_ptr<Domain2D> domain;
    std::unique_ptr<SpectralMask2D> mask;
    std::unique_ptr<State> state;
    std::unique_ptr<Thermodynamics> thermo;
    std::unique_ptr<FreeEnergy> free_energy;
    std::unique_ptr<TransportCoefficient> transport;
    std::unique_ptr<FCalculator> fcalc;
    std::unique_ptr<TimeIntegrator> integrator;
    RHSOperators rhs;
    // measures of the script (absent when it has none)
    std::unique_ptr<MeasureRegistry> measure_registry;
    std::unique_ptr<FourierTransform2D> fft;
    std::unique_ptr<MeasurementManager> measures;
    bool srk3 = true;
    double time = 0.0;
    long step = 0;

    // noise capture: [slot a|b][field][spectral] complex, filled during one step
    std::vector<Complex> noise;
    int psi_calls = 0;
    int j_calls = 0;
};

void parse_script_text(Params& params, const std::string& text) {
    char path[] = "/tmp/shhd_ref_scriptXXXXXX";
    const int fd = mkstemp(path);
    if (fd < 0) throw std::runtime_error("cannot create temporary script file");
    {
        std::ofstream out(path);
        out << text;
    }
    close(fd);
    ThermodynamicsRegistry thermo_registry = build_thermodynamics_registry();
    FreeEnergyRegistry free_energy_registry = build_free_energy_registry();
    TransportCoefficientRegistry transport_registry = build_transport_coefficient_registry();
    MeasureRegistry measure_registry = build_measure_registry();
    InitialConditionRegistry initial_registry = build_initial_condition_registry();
    ParamParser parser(params, thermo_registry, free_energy_registry, transport_registry, measure_registry, initial_registry);
    try {
        parser.parse_file(path);
    } catch (...) {
        unlink(path);
        throw;
    }
    unlink(path);
}

std::unique_ptr<TimeIntegrator> make_integrator(const Params& params, const Domain2D& domain, const SpectralMask2D& mask, bool& srk3) {
    const std::string& type = params.runtime.time_evolution_type;
    srk3 = type.rfind("srk3/", 0) == 0;
    if (type == "euler/compressible") return std::make_unique<EulerCompressible>(domain, params, mask);
    if (type == "euler/quiescent") return std::make_unique<EulerQuiescent>(domain, params, mask);
    if (type == "euler/incompressible") return std::make_unique<EulerIncompressible>(domain, params, mask);
    if (type == "srk3/compressible") return std::make_unique<SRK3Compressible>(domain, params, mask);
    if (type == "srk3/quiescent") return std::make_unique<SRK3Quiescent>(domain, params, mask);
    if (type == "srk3/incompressible") return std::make_unique<SRK3Incompressible>(domain, params, mask);
    throw std::runtime_error("unknown time_evolution type: " + type);
}

void build(RefRun& r) {
    r.domain = std::make_unique<Domain2D>(r.params);
    r.mask = std::make_unique<SpectralMask2D>(r.params, *r.domain);
    r.state = std::make_unique<State>(r.params, *r.domain);

    if (r.params.physics.thermo) {
        ThermodynamicsRegistry reg = build_thermodynamics_registry();
        r.thermo = reg.get_thermo(r.params.physics.thermo->type).create(r.params, r.params.physics.thermo);
    } else {
        r.thermo = std::make_unique<NullThermodynamics>();
    }
    if (r.params.physics.free_energy) {
        FreeEnergyRegistry reg = build_free_energy_registry();
        r.free_energy = reg.get_free_energy(r.params.physics.free_energy->type).create(r.params, r.params.physics.free_energy);
    } else {
        r.free_energy = std::make_unique<NullFreeEnergy>(r.params.physics.num_order_parameters);
    }
    if (!r.params.physics.transport) throw std::runtime_error("Project requires model transport.");
    {
        TransportCoefficientRegistry reg = build_transport_coefficient_registry();
        r.transport = reg.get_transport(r.params.physics.transport->type).create(r.params, r.params.physics.transport);
    }

    // initial conditions, as Project::apply_initial_conditions
    InitialConditionRegistry icr = build_initial_condition_registry();
    r.state->clear();
    for (const auto& c : r.params.initial.density_commands)
        icr.get_density(c->type).create_initial_condition(r.params, c)->apply(*r.state, *r.domain, *r.mask);
    for (const auto& c : r.params.initial.momentum_commands)
        icr.get_momentum(c->type).create_initial_condition(r.params, c)->apply(*r.state, *r.domain, *r.mask);
    for (const auto& c : r.params.initial.order_parameter_commands)
        icr.get_order_parameter(c->type).create_initial_condition(r.params, c)->apply(*r.state, *r.domain, *r.mask);
    if (is_incompressible_mode(parse_dynamics_mode(r.params.runtime.time_evolution_type)))
        validate_initial_momentum_is_transverse(*r.state, *r.domain, *r.mask);

    r.fcalc = std::make_unique<FCalculator>(r.params, *r.domain, *r.mask, *r.thermo, *r.free_energy, *r.transport);
    r.integrator = make_integrator(r.params, *r.domain, *r.mask, r.srk3);

    bool any_measure = false;
    for (const auto& c : r.params.commands) any_measure |= c.type == Command::Type::Measure;
    if (any_measure) {
        r.measure_registry = std::make_unique<MeasureRegistry>(build_measure_registry());
        r.fft = std::make_unique<FourierTransform2D>(*r.domain);
        r.measures = std::make_unique<MeasurementManager>(r.params, *r.domain, *r.measure_registry, *r.thermo, *r.free_energy,
                                                          *r.transport);
        for (const auto& c : r.params.commands)
            if (c.type == Command::Type::Measure) r.measures->apply_measure_command(c.measure);
        r.integrator->set_flux_request(r.measures->flux_request());
    }

    const std::size_t nspec = r.domain->spectral_size();
    const int nfields = r.params.physics.num_order_parameters + 3;
    r.noise.assign(2 * static_cast<std::size_t>(nfields) * nspec, Complex(0.0, 0.0));

    FCalculator* fc = r.fcalc.get();
    RefRun* rp = &r;
    r.rhs.rho_det = [fc](const State& s, Complex* out, double t, FluxBuffer* f) { fc->rho_det(s, out, t, f); };
    r.rhs.psi_det = [fc](int op, const State& s, Complex* out, double t, FluxBuffer* f) { fc->psi_det(op, s, out, t, f); };
    r.rhs.j_det = [fc](const State& s, Complex* ox, Complex* oy, double t, FluxBuffer* f) { fc->j_det(s, ox, oy, t, f); };

    // same binding rule as fluid_solver.h:79-94, plus a copy of each draw
    if (r.params.fix.noise.enabled) {
        if (r.params.fix.noise.order_parameter_enabled && r.params.physics.num_order_parameters > 0) {
            r.rhs.psi_sto = [fc, rp, nspec, nfields](int op, const State& s, Complex* out, FluxBuffer* f) {
                fc->psi_sto(op, s, out, f);
                const int slot = rp->srk3 ? (rp->psi_calls % 2) : 0;
                ++rp->psi_calls;
                Complex* dst = rp->noise.data() + (static_cast<std::size_t>(slot) * nfields + (op + 1)) * nspec;
                std::memcpy(dst, out, nspec * sizeof(Complex));
            };
        }
        const bool quiescent = r.params.runtime.time_evolution_type == "euler/quiescent" ||
                               r.params.runtime.time_evolution_type == "srk3/quiescent";
        if (r.params.fix.noise.momentum_enabled && !quiescent) {
            const int q = r.params.physics.num_order_parameters;
            r.rhs.j_sto = [fc, rp, nspec, nfields, q](const State& s, Complex* ox, Complex* oy, FluxBuffer* f) {
                fc->j_sto(s, ox, oy, f);
                const int slot = rp->srk3 ? (rp->j_calls % 2) : 0;
                ++rp->j_calls;
                Complex* dx = rp->noise.data() + (static_cast<std::size_t>(slot) * nfields + (q + 1)) * nspec;
                std::memcpy(dx, ox, nspec * sizeof(Complex));
                std::memcpy(dx + nspec, oy, nspec * sizeof(Complex));
            };
        }
    }
}

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

} // namespace

bool shref_view(void* handle, RefRunView& out) {
    if (!handle) return false;
    RefRun* r = static_cast<RefRun*>(handle);
    out.params = &r->params;
    out.domain = r->domain.get();
    out.thermodynamics = r->thermo.get();
    out.free_energy = r->free_energy.get();
    out.transport = r->transport.get();
    out.state = r->state.get();
    return true;
}

extern "C" {

const char* shref_last_error() { return g_error.c_str(); }

void* shref_create(const char* script_text) {
    RefRun* r = new RefRun();
    const int rc = guarded([&] {
        parse_script_text(r->params, script_text);
        build(*r);
    });
    if (rc != 0) {
        delete r;
        return nullptr;
    }
    return r;
}

void shref_destroy(void* h) { delete static_cast<RefRun*>(h); }

/* info[0..9] = nx, ny (compute), active nx, ny, nfields, num_order_parameters,
 * spectral_size, physical_size, srk3 flag, mode (0 compressible, 1 incompressible, 2 quiescent) */
int shref_info(void* h, long* info, double* dinfo) {
    RefRun* r = static_cast<RefRun*>(h);
    info[0] = r->domain->nx_global();
    info[1] = r->domain->ny_global();
    info[2] = r->params.grid.active_num_grid[0];
    info[3] = r->params.grid.active_num_grid[1];
    info[4] = r->params.physics.num_order_parameters + 3;
    info[5] = r->params.physics.num_order_parameters;
    info[6] = static_cast<long>(r->domain->spectral_size());
    info[7] = static_cast<long>(r->domain->physical_size());
    info[8] = r->srk3 ? 1 : 0;
    const DynamicsMode m = parse_dynamics_mode(r->params.runtime.time_evolution_type);
    info[9] = is_compressible_mode(m) ? 0 : (is_incompressible_mode(m) ? 1 : 2);
    dinfo[0] = r->domain->lx();
    dinfo[1] = r->domain->ly();
    dinfo[2] = r->params.runtime.dt;
    dinfo[3] = r->time;
    return 0;
}

int shref_get_state(void* h, double* out) {
    RefRun* r = static_cast<RefRun*>(h);
    const std::size_t n = static_cast<std::size_t>(r->state->num_fields()) * r->domain->spectral_size();
    std::memcpy(out, r->state->data(), n * sizeof(Complex));
    return 0;
}

int shref_set_state(void* h, const double* in) {
    RefRun* r = static_cast<RefRun*>(h);
    const std::size_t n = static_cast<std::size_t>(r->state->num_fields()) * r->domain->spectral_size();
    std::memcpy(r->state->data(), in, n * sizeof(Complex));
    return 0;
}

/* Advance nsteps.  If noise_out is non-null it receives, per step, the
 * stochastic RHS the integrator drew: [step][slot a,b][field][spectral]. */
int shref_step(void* h, int nsteps, double* noise_out) {
    RefRun* r = static_cast<RefRun*>(h);
    return guarded([&] {
        const std::size_t per_step = r->noise.size();
        for (int s = 0; s < nsteps; ++s) {
            std::fill(r->noise.begin(), r->noise.end(), Complex(0.0, 0.0));
            r->psi_calls = 0;
            r->j_calls = 0;
            r->integrator->step(*r->state, r->time, r->rhs);
            ++r->step;
            r->time += r->params.runtime.dt;
            if (r->measures)
                r->measures->observe(*r->state, *r->fft, r->integrator->flux_buffer(), static_cast<int>(r->step), r->time);
            if (noise_out) std::memcpy(noise_out + 2 * per_step * s, r->noise.data(), per_step * sizeof(Complex));
        }
    });
}

/* Close the files of the script's measures (MeasurementManager::finalize). */
int shref_finalize(void* h) {
    RefRun* r = static_cast<RefRun*>(h);
    return guarded([&] {
        if (r->measures) r->measures->finalize();
    });
}

/* Deterministic right-hand side at the current state, field order of State. */
int shref_rhs(void* h, double t, double* out) {
    RefRun* r = static_cast<RefRun*>(h);
    return guarded([&] {
        State det(r->params, *r->domain);
        det.clear();
        const DynamicsMode m = parse_dynamics_mode(r->params.runtime.time_evolution_type);
        // The workspace caches physical fields per (state address, time)
        // (fcalculator_workspace.cc:68-75); a NaN time never matches, so the
        // evaluation always sees the current state.  Time has no other use.
        (void)t;
        const double fresh = std::nan("");
        if (is_compressible_mode(m)) r->fcalc->rho_det(*r->state, det.rho_hat_data(), fresh, nullptr);
        for (int op = 0; op < r->params.physics.num_order_parameters; ++op)
            r->fcalc->psi_det(op, *r->state, det.psi_hat_data(op), fresh, nullptr);
        r->fcalc->j_det(*r->state, det.jx_hat_data(), det.jy_hat_data(), fresh, nullptr);
        const std::size_t n = static_cast<std::size_t>(det.num_fields()) * r->domain->spectral_size();
        std::memcpy(out, det.data(), n * sizeof(Complex));
    });
}

/* Host threads the shim transforms use. */
int shref_threads() { return shimfft::num_threads(); }

/* Wall time of nsteps steps (seconds), for the CPU baseline. */
double shref_time_steps(void* h, int nsteps) {
    RefRun* r = static_cast<RefRun*>(h);
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = guarded([&] {
        for (int s = 0; s < nsteps; ++s) {
            r->integrator->step(*r->state, r->time, r->rhs);
            ++r->step;
            r->time += r->params.runtime.dt;
        }
    });
    const auto t1 = std::chrono::steady_clock::now();
    if (rc != 0) return -1.0;
    return std::chrono::duration<double>(t1 - t0).count();
}

} // extern "C"
