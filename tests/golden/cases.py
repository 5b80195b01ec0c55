"""Input scripts of the golden cases (reference grammar).

Small grids so the fixtures stay a few hundred KB; together they reach every
term of the step: the three modes under Euler and SRK3, phi4 and quadratic
free energies, advection of psi and j, compressible and incompressible
viscosity, linear pressure, sine and gradient forces, the three dealias rules,
a rectangular box with an odd padded row count, and conservative noise.
"""

_HEAD = """dimension 2
boundary p p
"""

CASES = {
    # 1024^2 N=2 configuration shrunk to 16^2: compressible, phi4, advection, noise
    "srk3_compressible_n2": _HEAD + """grid 16 16
length 16 16
dealias 3/2
order_parameters 2
timestep 0.01
time_evolution srk3/compressible
model thermo linear_eos cT 1
model free_energy phi4 a[0] -1 b[0] 1 u[0] 1 a[1] -1 b[1] 1 u[1] 1
model transport constant eta 1 zeta 1 M[0,0] 1 M[1,1] 1
fix 1 all nonlinear on
fix 2 all noise on seed 3 kBT 1e-3
set density equilibrium/gaussian kBT 1e-3 rho0 1 cT 1 seed 1
set momentum all equilibrium/gaussian/compressible kBT 1e-3 seed 2
set order_parameter all equilibrium/gaussian seed 7 kBT 1 k0 4 k2 0
run 2
""",
    "euler_compressible_n2": _HEAD + """grid 16 16
length 16 16
dealias 3/2
order_parameters 2
timestep 0.005
time_evolution euler/compressible
model thermo linear_eos cT 1
model free_energy phi4 a[0] -1 b[0] 1 u[0] 1 a[1] 0.5 b[1] 2 u[1] 0
model transport constant eta 0.5 zeta 2 M[0,0] 1 M[1,1] 0.5
fix 1 all nonlinear on
fix 2 all noise on seed 11 kBT 1e-3 chi 2
set density equilibrium/gaussian kBT 1e-3 rho0 1 cT 1 seed 4
set momentum all equilibrium/gaussian/compressible kBT 1e-3 seed 5
set order_parameter all equilibrium/gaussian seed 9 kBT 1 k0 4 k2 0
run 2
""",
    "srk3_incompressible_n1_forces": _HEAD + """grid 16 16
length 12 12
dealias 3/2
order_parameters 1
timestep 0.01
time_evolution srk3/incompressible
model transport constant eta 0.3 zeta 0 M[0,0] 0.7
model free_energy phi4 a[0] 1 b[0] 0.5 u[0] 0.2
fix 1 all nonlinear on
fix 2 all noise on seed 5 kBT 1e-3
fix 3 momentum force/sine on component x axis y nk 2 amplitude 0.05
fix 4 order_parameter force/gradient on component 0 direction x amplitude 0.3
set density uniform value 1.3
set momentum all equilibrium/gaussian/incompressible kBT 1e-3 seed 3
set order_parameter all equilibrium/gaussian seed 2 kBT 1 k0 4 k2 0
run 2
""",
    "euler_incompressible_n0": _HEAD + """grid 16 16
length 16 16
dealias 3/2
order_parameters 0
timestep 0.01
time_evolution euler/incompressible
model transport constant eta 0.1 zeta 0
fix 1 momentum nonlinear on
fix 2 all noise on seed 8 kBT 1e-4
fix 3 momentum force/sine on component y axis x nk 3 amplitude 0.02
set density uniform value 1.0
set momentum all random_vorticity n0 3 sigma 2 urms 0.5 seed 11
run 2
""",
    # ensemble member shrunk to 16^2: quiescent phi4 quench with noise
    "srk3_quiescent_n1": _HEAD + """grid 16 16
length 16 16
dealias 3/2
order_parameters 1
timestep 0.02
time_evolution srk3/quiescent
model free_energy phi4 a[0] -1 b[0] 1 u[0] 1
model transport constant eta 0 zeta 0 M[0,0] 1
fix 1 order_parameter noise on seed 0 kBT 0.05
set density uniform value 1.0
set order_parameter all equilibrium/gaussian seed 0 kBT 0.01 k0 1 k2 0
run 2
""",
    "euler_quiescent_n2_quadratic": _HEAD + """grid 16 16
length 10 10
dealias 3/2
order_parameters 2
timestep 0.01
time_evolution euler/quiescent
model free_energy quadratic a[0] 1 a[1] 2.5
model transport constant eta 0 zeta 0 M[0,0] 1 M[1,1] 0.25
fix 1 order_parameter noise on seed 21 kBT 0.1
set density uniform value 1.0
set order_parameter all equilibrium/gaussian seed 4 kBT 0.1 k0 1 k2 1
run 2
""",
    # plain-method configuration shrunk: N=0 compressible, no dealiasing, rectangular box
    "srk3_compressible_n0_rect_nodealias": _HEAD + """grid 16 12
length 16 10
dealias none
order_parameters 0
timestep 0.02
time_evolution srk3/compressible
model thermo linear_eos cT 1
model transport constant eta 1 zeta 1
fix 1 all nonlinear on
fix 2 all noise on seed 1 kBT 1e-4
set density equilibrium/gaussian kBT 1e-4 rho0 1 cT 1 seed 1
set momentum all equilibrium/gaussian/compressible kBT 1e-4 seed 1
run 2
""",
    # dealias two, compressible gradient force, order-parameter sine force, odd padded rows (6 -> 9)
    "srk3_compressible_n1_two_gradient": _HEAD + """grid 12 6
length 9 7
dealias 3/2
order_parameters 1
timestep 0.005
time_evolution srk3/compressible
model thermo linear_eos cT 0.8
model free_energy phi4 a[0] 0.5 b[0] 0.3 u[0] 0.4
model transport constant eta 0.4 zeta 0.1 M[0,0] 0.6
fix 1 all nonlinear on
fix 2 all noise on seed 17 kBT 1e-3
fix 3 order_parameter force/gradient on component 0 direction y amplitude 0.2
fix 4 order_parameter force/sine on component 0 axis x nk 2 amplitude 0.1
set density equilibrium/gaussian kBT 1e-3 rho0 1 cT 0.8 seed 6
set momentum all equilibrium/gaussian/compressible kBT 1e-3 seed 7
set order_parameter all equilibrium/gaussian seed 8 kBT 1 k0 2 k2 0
run 2
""",
    "srk3_compressible_two_dealias": _HEAD + """grid 8 8
length 8 8
dealias two
order_parameters 1
timestep 0.01
time_evolution srk3/compressible
model thermo linear_eos cT 1
model free_energy phi4 a[0] -1 b[0] 1 u[0] 1
model transport constant eta 1 zeta 0.5 M[0,0] 1
fix 1 all nonlinear on
fix 2 all noise on seed 2 kBT 1e-3
set density equilibrium/gaussian kBT 1e-3 rho0 1 cT 1 seed 3
set momentum all equilibrium/gaussian/compressible kBT 1e-3 seed 4
set order_parameter all equilibrium/gaussian seed 5 kBT 1 k0 4 k2 0
run 2
""",
}


# Initial-condition-only cases: the state (or the error) the reference's `set`
# styles produce, recorded without stepping.  They reach every built-in style,
# the default seed, the `all` targets, last-command-wins and the parse / apply
# errors.
def _ic(grid, length, dealias, nop, te, sets, thermo=True):
    lines = [f"grid {grid[0]} {grid[1]}", f"length {length[0]} {length[1]}", f"dealias {dealias}",
             f"order_parameters {nop}", "timestep 0.01", f"time_evolution {te}"]
    if thermo:
        lines.append("model thermo linear_eos cT 1")
    if nop:
        lines.append("model free_energy phi4 " + " ".join(f"a[{i}] -1 b[{i}] 1 u[{i}] 1" for i in range(nop)))
    lines.append("model transport constant eta 1 zeta 1" + "".join(f" M[{i},{i}] 1" for i in range(nop)))
    return _HEAD + "\n".join(lines + sets) + "\nrun 1\n"


IC_CASES = {
    "bump_and_sine": _ic((16, 16), (16.0, 12.0), "3/2", 2, "srk3/compressible", [
        "set density gaussian base 1 amplitude 0.3 x0 3 y0 5 sigma 1.5",
        "set momentum x sine base 0.02 amplitude 0.1 nkx 2 nky -3",
        "set momentum y sine base 0 amplitude 0.05 nkx 0 nky -2",
        "set order_parameter 0 gaussian base 0.1 amplitude -0.2 x0 8 y0 2 sigma_x 2 sigma_y 1",
        "set order_parameter 1 sine amplitude 0.4 nkx 0 nky 3",
    ]),
    "default_seeds_rect": _ic((20, 12), (20.0, 9.0), "two", 1, "euler/compressible", [
        "set density sine base 1 amplitude 0.5 nkx 3",
        "set density equilibrium/gaussian kBT 2e-3 rho0 1.2 cT 0.9",
        "set momentum all equilibrium/gaussian/compressible kBT 1e-3",
        "set order_parameter all equilibrium/gaussian kBT 0.5 k0 1 k2 1 k4 0.25 psi0 -0.1",
    ]),
    "vorticity_on_bump_density": _ic((16, 16), (10.0, 10.0), "3/2", 1, "srk3/incompressible", [
        "set density gaussian base 1.1 amplitude 0.2 x0 5 y0 5 sigma 2",
        "set momentum all random_vorticity n0 2.5 sigma 1.2 urms 0.3",
        "set order_parameter 0 equilibrium/gaussian seed 9 kBT 1 k0 4 k2 0",
        "set order_parameter 0 uniform value 0.25",
    ], thermo=False),
    "incompressible_gaussian_default_seed": _ic((12, 16), (9.0, 12.0), "3/2", 0, "euler/incompressible", [
        "set density uniform value 0.8",
        "set momentum all equilibrium/gaussian/incompressible kBT 2e-3",
    ], thermo=False),
    "error_sine_density_base": _ic((16, 16), (16.0, 16.0), "3/2", 0, "srk3/compressible", [
        "set density sine base 0.1 amplitude 0.5 nkx 1",
    ]),
    "error_not_transverse": _ic((16, 16), (16.0, 16.0), "3/2", 0, "srk3/incompressible", [
        "set density uniform value 1",
        "set momentum all equilibrium/gaussian/compressible kBT 1e-3 seed 2",
    ], thermo=False),
    "error_x_replaced_not_transverse": _ic((16, 16), (16.0, 16.0), "3/2", 0, "srk3/incompressible", [
        "set density uniform value 1",
        "set momentum all equilibrium/gaussian/incompressible kBT 1e-3 seed 4",
        "set momentum x uniform value 0.01",
    ], thermo=False),
    "error_vorticity_zero_density": _ic((16, 16), (16.0, 16.0), "3/2", 0, "srk3/compressible", [
        "set momentum x random_vorticity n0 2 sigma 1 urms 0.1 seed 3",
    ]),
    "error_order_parameter_coefficient": _ic((16, 16), (16.0, 16.0), "3/2", 1, "srk3/compressible", [
        "set density uniform value 1",
        "set order_parameter 0 equilibrium/gaussian seed 1 kBT 1 k0 -1 k2 0",
    ]),
}


# Measure cases: a step case with the reference's own measures appended; the
# fixtures hold the state after every step and the text of every file the
# measures wrote (@DIR@ is replaced by a scratch directory when they are made).
_TS_ALL = "E_T E_K E_psi E_C pi_xx pi_xy pi_yy |rho|^2 |d_rho|^2 |j|^2 |d_j|^2"


def _measured(name, extra_targets, nsteps=3):
    body = CASES[name].rsplit("run ", 1)[0]
    return body + "\n".join([
        f"measure ts time_series on nevery 1 file @DIR@/ts.dat target {_TS_ALL} {extra_targets}".rstrip(),
        "measure sp snapshot on nevery 3 file @DIR@/phys space physical",
        "measure ss snapshot on nevery 3 file @DIR@/spec space spectral",
        f"run {nsteps}",
    ]) + "\n"


MEASURE_CASES = {
    "srk3_compressible_n2": _measured("srk3_compressible_n2",
                                      "|psi[0]|^2 |d_psi[0]|^2 |psi[1]|^2 |d_psi[1]|^2 Jpsi[0]_x Jpsi[0]_y Jpsi[1]_x Jpsi[1]_y"),
    "euler_compressible_n2": _measured("euler_compressible_n2", "|psi[1]|^2 Jpsi[1]_y"),
    "srk3_incompressible_n1_forces": _measured("srk3_incompressible_n1_forces", "|psi[0]|^2 |d_psi[0]|^2 Jpsi[0]_x"),
    "euler_quiescent_n2_quadratic": _measured("euler_quiescent_n2_quadratic", "|psi[0]|^2 |d_psi[1]|^2 Jpsi[0]_y"),
    "srk3_compressible_n0_rect_nodealias": _measured("srk3_compressible_n0_rect_nodealias", ""),
    "srk3_compressible_two_dealias": _measured("srk3_compressible_two_dealias", "Jpsi[0]_x"),
}


# ave/profile cases: both axes, block and running averages, nevery > 1, spectral
# targets and the compressible (physical-space) velocity; 6 steps each.
def _profiled(name, lines, nsteps=6):
    body = CASES[name].rsplit("run ", 1)[0]
    return body + "\n".join(lines + [f"run {nsteps}"]) + "\n"


PROFILE_CASES = {
    "profile_srk3_compressible_n2": _profiled("srk3_compressible_n2", [
        "measure p1 ave/profile on axis x nevery 1 nblock 3 file @DIR@/px_block.dat average block target rho jx vy psi[1] vx",
        "measure p2 ave/profile on axis y nevery 2 nblock 4 file @DIR@/py_running.dat average running target vx jy psi[0] rho",
    ]),
    "profile_srk3_incompressible_n1_forces": _profiled("srk3_incompressible_n1_forces", [
        "measure p1 ave/profile on axis y nevery 1 nblock 3 file @DIR@/py_block.dat average block target vx vy psi[0]",
        "measure p2 ave/profile on axis x nevery 1 nblock 2 file @DIR@/px_running.dat average running target jx rho vy",
    ]),
    "profile_euler_quiescent_n2_quadratic": _profiled("euler_quiescent_n2_quadratic", [
        "measure p1 ave/profile on axis x nevery 1 nblock 3 file @DIR@/px.dat average block target psi[0] psi[1] rho",
    ]),
    "profile_srk3_compressible_n0_rect_nodealias": _profiled("srk3_compressible_n0_rect_nodealias", [
        "measure p1 ave/profile on axis y nevery 1 nblock 2 file @DIR@/py.dat average running target vx vy rho jx",
    ]),
}


# ave/profile flux targets on noise-free copies of step cases (the reference's
# flux buffer then holds only the deterministic stage fluxes, which the engine
# reproduces without replaying the reference's noise); 6 steps each.
def _noiseless(name):
    return "\n".join(ln for ln in CASES[name].splitlines() if not (ln.startswith("fix") and " noise " in ln)) + "\n"


def _flux_profiled(name, lines, nsteps=6):
    body = _noiseless(name).rsplit("run ", 1)[0]
    return body + "\n".join(lines + [f"run {nsteps}"]) + "\n"


FLUX_PROFILE_CASES = {
    "fluxprof_srk3_compressible_n2": _flux_profiled("srk3_compressible_n2", [
        "measure p1 ave/profile on axis y nevery 1 nblock 3 file @DIR@/py_block.dat average block target pi_xx pi_xy pi_yy Jpsi[0]_x Jpsi[1]_y",
        "measure p2 ave/profile on axis x nevery 2 nblock 2 file @DIR@/px_running.dat average running target pixy Jpsi[0]_y piyy Jpsi[1]_x rho",
    ]),
    "fluxprof_srk3_incompressible_n1_forces": _flux_profiled("srk3_incompressible_n1_forces", [
        "measure p1 ave/profile on axis y nevery 1 nblock 3 file @DIR@/py_block.dat average block target vx pi_xy pi_xx pi_yy Jpsi[0]_y",
        "measure p2 ave/profile on axis x nevery 1 nblock 2 file @DIR@/px_running.dat average running target pi_xx Jpsi[0]_x pi_yy",
    ]),
    "fluxprof_euler_compressible_n2": _flux_profiled("euler_compressible_n2", [
        "measure p1 ave/profile on axis x nevery 1 nblock 3 file @DIR@/px_block.dat average block target pi_xx pi_xy pi_yy Jpsi[0]_x Jpsi[0]_y",
    ]),
    "fluxprof_euler_quiescent_n2_quadratic": _flux_profiled("euler_quiescent_n2_quadratic", [
        "measure p1 ave/profile on axis y nevery 1 nblock 2 file @DIR@/py.dat average running target Jpsi[0]_y Jpsi[1]_x psi[1]",
    ]),
}


# Yokota-Green-Kubo measure cases.  eta = zeta = 0 leaves the momentum without
# noise (j_sto returns early) and psi does not enter the momentum equations, so
# pi_xy, and with it every S_mean the reference writes, is deterministic while
# the measure still sees the positive kBT of `fix noise` it requires.  Grid
# spacing 2 keeps phi4's gradient term inside SRK3's stability interval.
def _gk_case(grid, length, lines, nsteps):
    return _HEAD + "\n".join([
        f"grid {grid[0]} {grid[1]}", f"length {length[0]} {length[1]}", "dealias 3/2", "order_parameters 1",
        "timestep 0.01", "time_evolution srk3/compressible", "model thermo linear_eos cT 1",
        "model free_energy phi4 a[0] -1 b[0] 1 u[0] 1", "model transport constant eta 0 zeta 0 M[0,0] 1",
        "fix 1 all nonlinear on", "fix 2 all noise on seed 5 kBT 1e-3",
        "set density equilibrium/gaussian kBT 1e-3 rho0 1 cT 1 seed 1",
        "set momentum all equilibrium/gaussian/compressible kBT 1e-3 seed 2",
        "set order_parameter all equilibrium/gaussian seed 3 kBT 1 k0 2 k2 0",
    ] + lines + [f"run {nsteps}"]) + "\n"


GK_CASES = {
    "gk_diagonal": _gk_case((16, 16), (32.0, 32.0), [
        "measure gk yokota_green_kubo on nevery 2 nblock 4 file @DIR@/gk.dat mode diagonal"], 8),
    "gk_all_rect": _gk_case((16, 12), (32.0, 18.0), [
        "measure gk yokota_green_kubo on nevery 1 nblock 3 file @DIR@/gk_all.dat mode all",
        "measure ts time_series on nevery 1 file @DIR@/ts.dat target E_K pi_xy"], 6),
}
