/*
 * shhd_b200_fluid_solver.hpp — reference-side drop-in for FluidSolver.
 *
 * A header for the reference solver's own source tree: it includes the
 * reference's headers (src/state.h, src/simulationinfo.h, the model headers)
 * and compiles only with that directory on the include path.  B200FluidSolver
 * has FluidSolver's constructor arguments and its step signature
 * (src/fluid_solver.h:52-99), so Project (src/project.h:148-177) keeps its
 * code and swaps the type:
 *
 *     B200FluidSolver solver(params, domain, thermodynamics, free_energy, transport);
 *     solver.step(state, time);             // FluidSolver::step(State&, double)
 *
 * The engine it drives is the C ABI of include/shhd_b200.h.  The configuration
 * is read from the same Params the reference parsed and from the model
 * objects through their public interface (model_free_energy.h:27-45,
 * model_thermodynamics.h:25-36, model_transport_coefficient.h:50-85); a model
 * the engine does not implement (a physical pressure or viscosity, or a
 * physical chemical potential that is not u psi_a^3) is refused with
 * std::runtime_error, the reference's error convention.
 *
 * Host synchronisation (set_host_sync): the reference's step reads and writes
 * the host State.  HostSync::every_step (the default) keeps exactly that:
 * upload before and download after each step, so any host-side change to the
 * State between steps is seen.  HostSync::download makes the device state
 * authoritative after the first upload and only refreshes the host State after
 * each step (measures that read it).  HostSync::resident refreshes it only on
 * fetch(); use it when nothing reads the State between steps.  Noise is the
 * engine's counter-based Philox stream keyed by the script's seed (the
 * reference draws mt19937_64), so noisy runs agree in distribution, and
 * noise-free runs agree with the reference's trajectory.
 */
#ifndef SHHD_B200_FLUID_SOLVER_HPP
#define SHHD_B200_FLUID_SOLVER_HPP

#include "domain.h"
#include "model_free_energy.h"
#include "model_thermodynamics.h"
#include "model_transport_coefficient.h"
#include "shhd_b200.h"
#include "simulationinfo.h"
#include "state.h"

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

class B200FluidSolver {
public:
    enum class HostSync { every_step, download, resident };

    B200FluidSolver(const Params& params, const Domain2D& domain, const Thermodynamics& thermodynamics, const FreeEnergy& free_energy,
                    const TransportCoefficient& transport_coefficient, int precision = SHHD_FP64) {
        (void)domain;  // the grid and box come from params.grid, as Domain2D's own constructor takes them
        shhd_config cfg = config_from(params, thermodynamics, free_energy, transport_coefficient);
        cfg.precision = precision;
        check(shhd_engine_create(&cfg, &engine_));
        shhd_info info;
        check(shhd_engine_info(engine_, &info));
        state_doubles_ = info.state_doubles;
    }
    B200FluidSolver(const B200FluidSolver&) = delete;
    B200FluidSolver& operator=(const B200FluidSolver&) = delete;
    ~B200FluidSolver() { shhd_engine_destroy(engine_); }

    // FluidSolver::step (src/fluid_solver.h:97-99); `time` only keys the reference's RHS cache
    // (fcalculator_workspace.cc:68-75), the engine keeps its own step counter
    void step(State& state, double time) {
        (void)time;
        if (sync_ == HostSync::every_step || !uploaded_) upload(state);
        check(shhd_engine_step(engine_, 1));
        if (sync_ != HostSync::resident) download(state);
    }

    void set_host_sync(HostSync mode) { sync_ = mode; }
    HostSync host_sync() const { return sync_; }

    // the device state into the host State (after resident steps)
    void fetch(State& state) { download(state); }
    // the host State into the device (after the host changed it under download / resident)
    void upload(const State& state) {
        check(shhd_engine_set_state(engine_, 0, reinterpret_cast<const double*>(state.data()), state_doubles_));
        uploaded_ = true;
    }

    shhd_engine* engine() const { return engine_; }

    // Params + models -> the engine configuration (the fields shhd_config_from_script fills)
    static shhd_config config_from(const Params& p, const Thermodynamics& th, const FreeEnergy& fe, const TransportCoefficient& tr) {
        if (th.has_physical_pressure()) throw std::runtime_error("B200FluidSolver: physical pressure models are not implemented.");
        if (tr.has_physical_shear_viscosity() || tr.has_physical_bulk_viscosity())
            throw std::runtime_error("B200FluidSolver: physical viscosity models are not implemented.");
        shhd_config c;
        check(shhd_config_default(&c));
        c.active_nx = p.grid.active_num_grid[0];
        c.active_ny = p.grid.active_num_grid[1];
        c.nx = p.grid.num_grid[0];
        c.ny = p.grid.num_grid[1];
        c.lx = p.grid.length[0];
        c.ly = p.grid.length[1];
        c.dt = p.runtime.dt;
        const std::string& te = p.runtime.time_evolution_type;
        const std::size_t slash = te.find('/');
        const std::string integ = te.substr(0, slash), mode = slash == std::string::npos ? "" : te.substr(slash + 1);
        if (integ == "euler") c.integrator = SHHD_EULER;
        else if (integ == "srk3") c.integrator = SHHD_SRK3;
        else throw std::runtime_error("unknown time_evolution type: " + te);
        if (mode == "compressible") c.mode = SHHD_COMPRESSIBLE;
        else if (mode == "incompressible") c.mode = SHHD_INCOMPRESSIBLE;
        else if (mode == "quiescent") c.mode = SHHD_QUIESCENT;
        else throw std::runtime_error("unknown time_evolution type: " + te);
        const int nop = p.physics.num_order_parameters;
        if (nop > SHHD_MAX_ORDER_PARAMETERS) throw std::runtime_error("B200FluidSolver: too many order parameters.");
        c.num_order_parameters = nop;
        // free energy: linear coefficients of mu, and the physical part probed as u psi_a^3
        const bool phys = nop > 0 && fe.has_physical_chemical_potential();
        c.free_energy = phys ? SHHD_FE_PHI4 : (nop > 0 ? SHHD_FE_QUADRATIC : SHHD_FE_NONE);
        for (int a = 0; a < nop; ++a) {
            c.mu_k0[a] = fe.chemical_potential_k0_coefficient(a);
            c.mu_k2[a] = fe.chemical_potential_k2_coefficient(a);
            c.mu_k4[a] = fe.chemical_potential_k4_coefficient(a);
            c.mu_u3[a] = 0.0;
            if (phys) {
                std::vector<double> psi(static_cast<std::size_t>(nop), 0.0);
                psi[static_cast<std::size_t>(a)] = 1.0;
                const double u = fe.physical_chemical_potential(a, psi.data());
                psi[static_cast<std::size_t>(a)] = 2.0;
                const double u8 = fe.physical_chemical_potential(a, psi.data());
                for (int b = 0; b < nop; ++b) psi[static_cast<std::size_t>(b)] = b == a ? 1.0 : 0.5;
                const double ux = fe.physical_chemical_potential(a, psi.data());
                if (std::fabs(u8 - 8.0 * u) > 1e-12 * std::fabs(8.0 * u) || std::fabs(ux - u) > 1e-12 * std::fabs(u))
                    throw std::runtime_error("B200FluidSolver: only the physical chemical potential u psi_a^3 is implemented.");
                c.mu_u3[a] = u;
            }
        }
        c.cT = std::sqrt(th.linear_pressure_coefficient());
        c.eta = tr.shear_viscosity();
        c.zeta = tr.bulk_viscosity();
        for (int a = 0; a < nop; ++a) c.mobility[a] = tr.order_parameter_mobility()[static_cast<std::size_t>(a)];
        c.momentum_advection = p.fix.momentum_advection ? 1 : 0;
        c.order_parameter_advection = p.fix.order_parameter_advection ? 1 : 0;
        const bool quiescent = c.mode == SHHD_QUIESCENT;
        c.noise_momentum = (p.fix.noise.enabled && p.fix.noise.momentum_enabled && !quiescent) ? 1 : 0;
        c.noise_order_parameter = (p.fix.noise.enabled && p.fix.noise.order_parameter_enabled && nop > 0) ? 1 : 0;
        c.noise_seed = p.fix.noise.seed;
        c.kBT = p.fix.noise.kBT;
        c.chi = p.fix.noise.order_parameter_noise_chi;
        c.n_sine_forces = 0;
        for (const SineForceFixConfig& f : p.fix.sine_forces) {
            if (!f.enabled) continue;
            if (c.n_sine_forces >= SHHD_MAX_FORCES) throw std::runtime_error("too many force/sine fixes");
            shhd_sine_force& s = c.sine_forces[c.n_sine_forces++];
            s.target = f.momentum_enabled ? 0 : 1;
            s.component = f.component;
            s.axis = f.axis;
            s.nk = f.nk;
            s.amplitude = f.amplitude;
        }
        c.n_gradient_forces = 0;
        for (const GradientForceFixConfig& f : p.fix.gradient_forces) {
            if (!f.enabled) continue;
            if (c.n_gradient_forces >= SHHD_MAX_FORCES) throw std::runtime_error("too many force/gradient fixes");
            shhd_gradient_force& g = c.gradient_forces[c.n_gradient_forces++];
            g.component = f.component;
            g.direction = f.direction;
            g.amplitude = f.amplitude;
        }
        c.noise_source = SHHD_NOISE_PHILOX;
        c.batch = 1;
        c.member_offset = 0;
        return c;
    }

private:
    static void check(int rc) {
        if (rc != SHHD_OK) throw std::runtime_error(shhd_last_error());
    }
    void download(State& state) { check(shhd_engine_get_state(engine_, 0, reinterpret_cast<double*>(state.data()), state_doubles_)); }

    shhd_engine* engine_ = nullptr;
    std::size_t state_doubles_ = 0;
    bool uploaded_ = false;
    HostSync sync_ = HostSync::every_step;
};

#endif /* SHHD_B200_FLUID_SOLVER_HPP */
