"""Pin the oracle against golden vectors produced by running the reference (CPU path).

Tolerances: FP32 oracle vs FP32 reference -- summation order differs (numpy vs torch), so
results agree to FP32 rounding: rel-L2 <= 5e-6 on residuals/gradients, <= 1e-6 on states.
FP64 oracle vs FP64 reference -- the oracle runs on FP32-built geometry, the FP64 reference on
FP64 geometry; rel-L2 <= 1e-4 on residuals, <= 1e-6 on states.
"""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import fvm_oracle as O


def test_residual_fp32(golden):
    g, spec, T, cfg = golden
    res = O.OracleResidual(T, cfg, np.float32)
    r1, g1 = res.forward(g["prim0"])
    assert rel_l2(r1, g["res1"]) < 5e-6
    assert rel_l2(g1, g["grads1"]) < 5e-6
    r2, g2 = res.forward(g["prim2"], g["grads1"])
    assert rel_l2(r2, g["res2"]) < 5e-6
    assert rel_l2(g2, g["grads2"]) < 5e-6


def test_residual_fp64(golden):
    g, spec, T, cfg = golden
    res = O.OracleResidual(T, cfg, np.float64)
    r1, g1 = res.forward(g["prim0"].astype(np.float64))
    assert rel_l2(r1, g["res1_f64"]) < 1e-4
    # FP32 reference is within its own rounding of the FP64 reference
    assert rel_l2(g["res1"], g["res1_f64"]) < 1e-4


@pytest.mark.parametrize("name,key", [("RK4", "rk4_step1"), ("SSP_RK3", "ssprk3_step1")])
def test_butcher_step(golden, name, key):
    g, spec, T, cfg = golden
    s = O.OracleSolver(O.OracleResidual(T, cfg, np.float32), g["state0"], float(g["dt"]))
    s.butcher_step(name)
    assert rel_l2(s.state, g[key]) < 1e-6
    s64 = O.OracleSolver(O.OracleResidual(T, cfg, np.float64), g["state0"].astype(np.float64), float(g["dt"]))
    s64.butcher_step(name)
    assert rel_l2(s64.state, g[key + "_f64"]) < 1e-6


def test_ten_steps(golden):
    g, spec, T, cfg = golden
    s = O.OracleSolver(O.OracleResidual(T, cfg, np.float32), g["state0"], float(g["dt"]))
    for _ in range(10):
        s.butcher_step("SSP_RK3")
    assert rel_l2(s.state, g["ssprk3_step10"]) < 2e-6


def test_adaptive_steps(golden):
    g, spec, T, cfg = golden
    s = O.OracleSolver(O.OracleResidual(T, cfg, np.float32), g["state0"], float(g["dt"]))
    s.adapt_step("RK3_SSP4")
    assert rel_l2(s.state, g["adapt_step1"]) < 1e-6
    assert abs(float(s.dt) / float(g["adapt_dt1"]) - 1) < 1e-5
    s = O.OracleSolver(O.OracleResidual(T, cfg, np.float32), g["state0"], float(g["dt"]))
    s.rk3ssp4_step()
    assert rel_l2(s.state, g["rk3ssp4_step1"]) < 1e-6
    assert abs(float(s.dt) / float(g["rk3ssp4_dt1"]) - 1) < 1e-5


@pytest.fixture(scope="module", params=["c2d11k", "b3d9k"])
def golden_light(request):
    from conftest import golden_setup
    return golden_setup(request.param)


def test_larger_mesh_residual(golden_light):
    """The oracle against the reference on the larger light fixtures (the 11 307-triangle channel
    mesh of the channel-cylinder benchmark, a 9 066-tet box): first residual in FP32 and FP64."""
    g, spec, T, cfg = golden_light
    r1, _ = O.OracleResidual(T, cfg, np.float32).forward(g["prim0"])
    assert rel_l2(r1, g["res1"]) < 5e-6
    r64, _ = O.OracleResidual(T, cfg, np.float64).forward(g["prim0"].astype(np.float64))
    assert rel_l2(r64, g["res1_f64"]) < 1e-4


def test_larger_mesh_ten_steps(golden_light):
    g, spec, T, cfg = golden_light
    s = O.OracleSolver(O.OracleResidual(T, cfg, np.float32), g["state0"], float(g["dt"]))
    for _ in range(10):
        s.butcher_step("SSP_RK3")
    assert rel_l2(s.state, g["ssprk3_step10"]) < 2e-6
    s64 = O.OracleSolver(O.OracleResidual(T, cfg, np.float64), g["state0"].astype(np.float64), float(g["dt"]))
    for _ in range(10):
        s64.butcher_step("SSP_RK3")
    assert rel_l2(s64.state, g["ssprk3_step10_f64"]) < 1e-6


# -- variants on the c2d mesh: limiters p1-p3, p5; tableaus RK3_SSP5/6, RK4_SSP5/10; AB3 ---------
@pytest.mark.parametrize("p", [1, 2, 3, 5])
def test_limiter_variants(p):
    """Limiter p (limiter.py:29-77) vs the reference: first residual and limited gradients, FP32
    bar 5e-6 as for the default limiter; FP64 oracle vs FP64 reference 1e-4 (FP32-built geometry)."""
    from conftest import golden_setup
    g, spec, T, cfg = golden_setup("c2dvar", lim_p=p)
    r1, g1 = O.OracleResidual(T, cfg, np.float32).forward(g["prim0"])
    assert rel_l2(r1, g[f"lim{p}_res1"]) < 5e-6
    assert rel_l2(g1, g[f"lim{p}_grads1"]) < 5e-6
    r64, _ = O.OracleResidual(T, cfg, np.float64).forward(g["prim0"].astype(np.float64))
    assert rel_l2(r64, g[f"lim{p}_res1_f64"]) < 1e-4


@pytest.mark.parametrize("name", ["RK3_SSP5", "RK3_SSP6", "RK4_SSP5", "RK4_SSP10"])
def test_tableau_variants(name):
    """One Butcher step with each remaining tableau (integrators.py:240-296): FP32 1e-6, FP64 1e-6."""
    from conftest import golden_setup
    g, spec, T, cfg = golden_setup("c2dvar")
    s = O.OracleSolver(O.OracleResidual(T, cfg, np.float32), g["state0"], float(g["dt"]))
    s.butcher_step(name)
    assert rel_l2(s.state, g[f"{name.lower()}_step1"]) < 1e-6
    s64 = O.OracleSolver(O.OracleResidual(T, cfg, np.float64), g["state0"].astype(np.float64), float(g["dt"]))
    s64.butcher_step(name)
    assert rel_l2(s64.state, g[f"{name.lower()}_step1_f64"]) < 1e-6


def test_ab3_vs_reference_residual():
    """AB3 (two SSP-RK3 start-up steps + three AB3 steps) against the same scheme driven by the
    reference's own residual: FP32 1e-6, FP64 1e-6."""
    from conftest import golden_setup
    g, spec, T, cfg = golden_setup("c2dvar")
    for dt_, key in ((np.float32, "ab3_step5"), (np.float64, "ab3_step5_f64")):
        s = O.OracleSolver(O.OracleResidual(T, cfg, dt_), g["state0"].astype(dt_), float(g["dt"]))
        s.ab3_start()
        for _ in range(3):
            s.ab3_step()
        assert rel_l2(s.state, g[key]) < 1e-6


# -- periodic Taylor-Green box vs the reference on the unrolled (3 x 3 x 3) mesh -----------------
def test_periodic_box_vs_unrolled_reference():
    """The periodic table build (wrapped displacements, LSQ offsets, facet pairing) against the
    reference's own geometry: the central tile of the unrolled box.  Residual 5e-6 and RK4 step
    1e-6 as on the other fixtures; limited gradients 1e-5, because the unrolled mesh numbers its
    cells and facets differently and the limiter amplifies the changed summation order (measured
    4.6e-6 here, the same in cells that wrap and cells that do not)."""
    from conftest import golden_setup
    g, spec, T, cfg = golden_setup("ptile")
    res = O.OracleResidual(T, cfg, np.float32)
    r1, g1 = res.forward(g["prim0"])
    assert rel_l2(r1, g["res1"]) < 5e-6
    assert rel_l2(g1, g["grads1"]) < 1e-5
    s = O.OracleSolver(res, g["state0"], float(g["dt"]))
    s.butcher_step("RK4")
    assert rel_l2(s.state, g["rk4_step1"]) < 1e-6
    s64 = O.OracleSolver(O.OracleResidual(T, cfg, np.float64), g["state0"].astype(np.float64), float(g["dt"]))
    s64.butcher_step("RK4")
    assert rel_l2(s64.state, g["rk4_step1_f64"]) < 1e-6
