"""The oracle's MTK NPT (src/cpu/dynamics/nose_hoover_npt.cpp), pinned to
the reference's own regression and checked for the properties of the
integrator (CPU only):

- regressions/md/npt_lj_mtk (REFERENCE.md): 6^3 simple-cubic LJ at
  rho = 0.8, T* = 1 (T = 1/k_B K with eps = 1 eV), tau_T = 0.1, P = 0,
  tau_P = 1, dt = 0.005, 80 steps, no force pass before the first step;
  the reference CPU build ends at V = 269.425432;
- tests/cuda/dynamics/test_nose_hoover_npt.cu: the first step moves the
  cell;
- the extended Hamiltonian fluctuates as dt^2 (second-order splitting);
- all-axes coupling keeps a cubic cell cubic (couple() averages the three
  axis pressures); an uncoupled axis keeps its edge; the temperature ramp
  follows compute_temp_target;
- with PME the influence tables follow the cell: forces after NPT steps
  equal a fresh evaluation in the final cell.
"""
import numpy as np
import pytest

KB = 8.617333262e-5


def lj_cube(n_side=6, rho=0.8):
    n = n_side ** 3
    L = (n / rho) ** (1.0 / 3.0)
    a = L / n_side
    idx = np.array([(ix, iy, iz) for ix in range(n_side) for iy in range(n_side)
                    for iz in range(n_side)])
    pos = (idx + 0.5) * a
    ix, iy, iz = idx[:, 0], idx[:, 1], idx[:, 2]
    v = np.stack([0.02 * ((ix + iy + iz) % 3 - 1), 0.02 * ((ix + 2 * iy) % 3 - 1),
                  0.02 * ((2 * ix + iz) % 3 - 1)], axis=1).astype(np.float64)
    return n, L, pos, v


def _lj_npt(orc, dt=0.005, tau_T=0.1, tau_P=1.0, setup=False, **npt):
    n, L, pos, v = lj_cube()
    d = orc.make_desc(n, (L, L, L), nl_cutoff=2.5, skin=0.3, has_lj=1, lj_eps=1.0,
                      lj_sigma=1.0, lj_rc=2.5, dt=dt)
    s = orc.OracleSystem(d)
    s.set_state(pos[:, 0], pos[:, 1], pos[:, 2], v[:, 0], v[:, 1], v[:, 2], mass=np.ones(n))
    s.set_npt(1.0 / KB, tau_T, 0.0, tau_P, **npt)
    if setup:
        s.build_list()
        s.compute_forces()
    return s, L ** 3


def test_mtk_lj_volume_pins_reference(orc):
    s, V0 = _lj_npt(orc)
    s.run(1)
    V1 = float(np.prod(s.npt_state()["box"]))
    assert abs(V1 - V0) > 1e-12          # the barostat moved the cell
    s.run(79)
    V = float(np.prod(s.npt_state()["box"]))
    assert V == pytest.approx(269.425432, abs=1e-6)
    assert np.isfinite(s.npt_state()["conserved"])


def test_mtk_extended_hamiltonian_is_second_order(orc):
    spread = []
    for dt in (0.005, 0.0025):
        s, _ = _lj_npt(orc, dt=dt, tau_T=0.5, tau_P=5.0, setup=True)
        H = []
        for _ in range(int(round(1.0 / dt))):
            s.run(1)
            H.append(s.npt_state()["conserved"])
        spread.append(np.ptp(H))
    assert spread[0] / abs(H[0]) < 1e-4
    assert 3.0 < spread[0] / spread[1] < 5.0


def test_isotropic_cell_stays_cubic_and_rigid_axis_keeps_edge(orc):
    s, _ = _lj_npt(orc, setup=True)
    s.run(20)
    b = s.npt_state()["box"]
    assert b[0] == b[1] == b[2]
    n, L, _, _ = lj_cube()
    s2, _ = _lj_npt(orc, setup=True, couple=(True, True, False))
    s2.run(20)
    b2 = s2.npt_state()["box"]
    assert b2[2] == L
    assert b2[0] != L and b2[1] != L      # pdim = 2: each axis on its own stress
    assert s2.npt_state()["eps_dot"][2] == 0.0


def test_temperature_ramp_follows_run_span(orc):
    T0, T1 = 1.0 / KB, 2.0 / KB
    s, _ = _lj_npt(orc, T_stop=T1, span=(0, 100))
    for k in range(5):
        s.run(1)
        # compute_temp_target at the step just taken (index k)
        assert s.npt_state()["T_live"] == pytest.approx(T0 + k / 100.0 * (T1 - T0), rel=1e-15)


def test_bad_parameters_rejected(orc):
    s, _ = _lj_npt(orc)
    with pytest.raises(ValueError):
        s.set_npt(300.0, 0.0, 0.0, 1.0)
    with pytest.raises(ValueError):
        s.set_npt(300.0, 1.0, 0.0, 1.0, mtchain=0)


def test_pme_tables_follow_the_cell(orc):
    from atomiverse_b200 import workloads as W
    desc, frame = W.rocksalt_melt(ncell=4, rc=5.5, grid=(16, 16, 16))
    n = desc["n_atoms"]
    L = desc["box"][0]
    kw = dict(nl_cutoff=desc["nl_cutoff"], skin=desc["nl_skin"], has_lj=1,
              lj_eps=desc["lj_epsilon"], lj_sigma=desc["lj_sigma"], lj_rc=desc["lj_cutoff"],
              has_coul=1, coul_alpha=desc["coul_alpha"], coul_rc=desc["coul_cutoff"],
              has_pme=1, pme_alpha=desc["pme_alpha"], pme_K=desc["pme_grid"], pme_order=4,
              dt=2.0)
    s = orc.OracleSystem(orc.make_desc(n, (L, L, L), **kw))
    s.set_state(frame["x"], frame["y"], frame["z"], frame["vx"], frame["vy"], frame["vz"],
                mass=frame["mass"], q=frame["charge"])
    s.set_npt(1200.0, 100.0, 1e-5, 1000.0)   # 1e-5 eV/A^3 ~ 16 kbar
    s.build_list()
    s.compute_forces()
    s.run(10)
    st = s.state()
    box = s.npt_state()["box"]
    assert box[0] != L
    fresh = orc.OracleSystem(orc.make_desc(n, tuple(box), **kw))
    fresh.set_state(st["x"], st["y"], st["z"], mass=frame["mass"], q=frame["charge"])
    fresh.build_list()
    fresh.compute_forces()
    f1 = fresh.state()
    for k in ("fx", "fy", "fz"):
        assert np.array_equal(st[k], f1[k])
    # energies: OpenMP reduction order may differ in the last bit
    assert fresh.scalars()["e_recip"] == pytest.approx(s.scalars()["e_recip"], rel=1e-14)


def _lj_baro(orc, P, thermostat=1):
    from atomiverse_b200 import workloads as W
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from conftest import oracle_system
    desc, frame = W.lj_fcc(ncell=5, t_star=1.0, seed=3, thermostat=thermostat)
    o = oracle_system(orc, dict(desc, tau=50.0), frame)
    o.set_barostat(P, 20.0, 10.0)
    o.build_list()
    o.compute_forces()
    return o, desc


def test_berendsen_one_step_dilation(orc):
    """barostat.cpp:27-110: after one step the cell is the old one times
    cbrt(1 - dt/(tau_P beta) (P_target - P)), P = (trace W + 2 KE)/(3 V) of
    that step's end."""
    o, desc = _lj_baro(orc, 0.5)
    L0 = desc["box"][0]
    o.run(1)
    sc = o.scalars()
    P = (sc["virial"][:3].sum() + 2.0 * sc["kinetic"]) / (3.0 * L0 ** 3)
    mu = np.cbrt(1.0 - desc["dt"] / (20.0 * 10.0) * (0.5 - P))
    assert o.npt_state()["box"][0] == pytest.approx(L0 * mu, rel=1e-15)


def test_berendsen_moves_the_cell_toward_the_target(orc):
    for P, sign in ((20.0, -1), (-20.0, 1)):
        o, desc = _lj_baro(orc, P)
        o.run(50)
        dL = o.npt_state()["box"][0] - desc["box"][0]
        assert np.sign(dL) == sign
    with pytest.raises(ValueError):
        o.set_barostat(0.0, 0.0, 1.0)


def test_deform_follows_engineering_strain(orc):
    """deform.cu:55-95: after k steps the edge is L0 (1 + rate dt k)."""
    from atomiverse_b200 import workloads as W
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from conftest import oracle_system
    desc, frame = W.lj_fcc(ncell=5, t_star=1.0, seed=3)
    o = oracle_system(orc, desc, frame)
    rate = 2e-3
    o.set_deform(2, rate)
    o.build_list()
    o.compute_forces()
    o.run(40)
    L = o.npt_state()["box"]
    L0 = desc["box"][0]
    assert L[2] == pytest.approx(L0 * (1.0 + rate * desc["dt"] * 40), rel=1e-13)
    assert L[0] == L0 and L[1] == L0
    with pytest.raises(ValueError):
        o.set_deform(3, rate)


def test_nve_limit_caps_speeds(orc):
    """nve_limit.cu:20-30: no atom moves faster than xmax / dt."""
    from atomiverse_b200 import workloads as W
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from conftest import oracle_system
    desc, frame = W.lj_fcc(ncell=5, t_star=3.0, seed=3)
    o = oracle_system(orc, desc, frame)
    xmax = 0.002
    o.set_nve_limit(xmax)
    o.build_list()
    o.compute_forces()
    o.run(5)
    st = o.state()
    v = np.sqrt(st["vx"] ** 2 + st["vy"] ** 2 + st["vz"] ** 2)
    vmax = xmax / desc["dt"]
    assert v.max() <= vmax * (1 + 1e-12)
    assert v.max() > 0.99 * vmax                  # the cap was active
