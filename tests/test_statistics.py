"""Statistical parity with the reference's own known answers (GPU, batched members).

* Equipartition: the reference's equilibrium example (examples/01_best_timestep_equilibrium,
  README.md:40-52 and plot_results.py:53-70): a 64^2 grid, 3/2 rule, compressible, one order
  parameter with quadratic free energy a = 1, linear EOS cT = 10, eta = zeta = M = 8, kBT = 1,
  relaxing from zero fluctuations.  Each nonzero active mode carries kBT / 2 per real degree of
  freedom: E_psi = E_C = 1984, E_K = 3968, E_T = 7936 (3968 degrees of freedom).  The time step
  is 0.001, below the example's stability table (dt <= 0.002 for this transport).
* Green-Kubo viscosity: the reference's Yokota-Green-Kubo example
  (examples/05_yokota_green_kubo/input_ohtaka_linear_sample.template, estimate_viscosity.py):
  16^2, no dealiasing, linear incompressible momentum with noise, eta = 0.1, kBT = 1,
  equilibrium initial momentum; measure every 100 steps in blocks of 10000 over diagonal modes.
  The long-tau value of S_mean is the viscosity, eta = 0.1, for every mode.

Members of one batched engine are independent realisations (their own noise keys and initial
seeds), so the error bars are the spread over members.  Both run the FP32 engine (FP64 sums).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EQUILIBRIUM = """dimension 2
grid 64 64
length 64.0 64.0
dealias three_halves
order_parameters 1
timestep 0.001
time_evolution srk3/compressible
model thermo linear_eos cT 10.0
model free_energy quadratic a[0] 1.0
model transport constant eta 8.0 zeta 8.0 M[0,0] 8.0
fix 1 all noise on seed 12345 kBT 1.0
fix 2 all nonlinear on
set density uniform value 1.0
set momentum all uniform value 0.0
set order_parameter all uniform value 0.0
run 10000
"""

GREEN_KUBO = """dimension 2
grid 16 16
length 16.0 16.0
dealias none
order_parameters 0
timestep 0.01
time_evolution srk3/incompressible
model transport constant eta 0.1 zeta 0.0
fix 1 momentum nonlinear off
fix 2 momentum noise on seed 7 kBT 1.0
set density uniform value 1.0
set momentum all equilibrium/gaussian/incompressible kBT 1.0 seed 3
run 100000
"""


def scalar_dof(nx, ny):
    """Real degrees of freedom of one scalar field over the nonzero active modes (the kx = 0
    line counts once per mode, the rest twice)."""
    return sum((1 if gx == 0 else 2) for gx in range(nx // 2) for ky in range(-(ny // 2) + 1, ny // 2) if (gx, ky) != (0, 0))


def test_equipartition_energies():
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state_device
    half = 0.5 * scalar_dof(64, 64) * 1.0
    theory = {"E_T": 4 * half, "E_K": 2 * half, "E_psi": half, "E_C": half}
    assert theory == {"E_T": 7936.0, "E_K": 3968.0, "E_psi": 1984.0, "E_C": 1984.0}
    cfg = sb.config_from_script(EQUILIBRIUM)
    cfg.precision = sb.FP32
    cfg.batch = 64
    with sb.Engine(cfg) as eng:
        eng.set_graph_chunk(100)
        for m in range(cfg.batch):
            initial_state_device(eng, EQUILIBRIUM, member=m)
        eng.step(6000)  # relaxation: the slowest modes decay at 2 M k_min^2 ~ 0.15 per time unit
        samples = []
        for _ in range(30):
            eng.step(100)
            samples.append([[eng.time_series_energies(m)[k] for k in theory] for m in range(cfg.batch)])
    a = np.array(samples)                      # [sample, member, column]
    per_member = a.mean(axis=0)
    mean = per_member.mean(axis=0)
    se = per_member.std(axis=0, ddof=1) / np.sqrt(cfg.batch)
    for c, (k, want) in enumerate(theory.items()):
        print(f"{k}: {mean[c]:.2f} +- {se[c]:.2f} (equipartition {want:.0f})")
        # statistical error plus 0.2% for the time step's bias
        assert abs(mean[c] - want) < 4 * se[c] + 2e-3 * want, (k, mean[c], se[c], want)


def test_green_kubo_viscosity():
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state_device
    eta = 0.1
    cfg = sb.config_from_script(GREEN_KUBO)
    cfg.precision = sb.FP32
    cfg.batch = 128
    with sb.Engine(cfg) as eng:
        eng.set_graph_chunk(500)
        for m in range(cfg.batch):
            initial_state_device(eng, GREEN_KUBO.replace("kBT 1.0 seed 3", f"kBT 1.0 seed {100 + m}"), member=m)
        eng.gk_enable(100, 10000, "diagonal")
        eng.step(100000)
        S = []
        for m in range(cfg.batch):
            sums, blocks = eng.gk_read(m)
            assert blocks == 10
            S.append(sums / blocks)
        modes = eng.gk_modes
    S = np.array(S)                             # [member, tau, mode]; tau = 1, 2, ..., 100
    tail = S[:, 69:, :].mean(axis=1)            # long-tau plateau: tau in [70, 100]
    mean = tail.mean(axis=0)
    se = tail.std(axis=0, ddof=1) / np.sqrt(cfg.batch)
    for q, (g, _) in enumerate(modes):
        print(f"mode ({g},{g}): S_mean plateau {mean[q]:.4f} +- {se[q]:.4f} (eta {eta})")
        assert abs(mean[q] - eta) < 4 * se[q], (modes[q], mean[q], se[q])
    est = mean.mean()
    est_se = np.sqrt((se ** 2).sum()) / len(modes)
    print(f"eta estimate over modes: {est:.4f} +- {est_se:.4f}")
    assert abs(est - eta) < 4 * est_se
