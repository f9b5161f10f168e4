"""Device equilibration (sankhya_b200_scale_factors) against the reference and the oracle.

pow2: c/src/sk_scale.c:20-72 (fixtures from the reference's own sk_scale_model, bit-exact).
Ruiz: src/lp/Scaling.cpp:11-92 (max-based, so bit-exact against the oracle).
Ruiz then Pock-Chambolle composed as src/lp/LpSolver.cpp:62-71 (sums in a different
order on the device: 1e-13 relative)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_pow2_bit_exact_vs_reference_fixture(engine, instances, golden_dir):
    man = json.load(open(os.path.join(golden_dir, "manifest.json")))
    for name, seed, m, n, per_col, _ in man["lp"]:
        inst = instances.lp_uniform(seed, m, n, per_col)
        g = np.load(os.path.join(golden_dir, f"sk_scale_{name}.npz"))
        A = engine.Matrix.from_instance(inst)
        rc, r, c = engine.scale_factors(A, engine.SCALE_POW2)
        assert rc == 0
        assert np.array_equal(r, g["R"]) and np.array_equal(c, g["C"])


@pytest.mark.parametrize("seed", [5, 6])
def test_ruiz_bit_exact_vs_oracle(engine, oracle, instances, seed):
    inst = instances.lp_powerlaw(seed, 3000, 6000, 60000)
    A = engine.Matrix.from_instance(inst)
    rc, r, c = engine.scale_factors(A, engine.SCALE_RUIZ, 100, 1e-2)
    ro, co, conv = oracle.ruiz(inst, 100, 1e-2)
    assert rc == 0 and conv
    assert np.array_equal(r, ro) and np.array_equal(c, co)
    # not converged within the budget: identity
    rc, r1, c1 = engine.scale_factors(A, engine.SCALE_RUIZ, 1, 1e-12)
    assert rc == 0 and np.all(r1 == 1.0) and np.all(c1 == 1.0)


def test_ruiz_then_pock_chambolle_vs_oracle(engine, oracle, instances):
    inst = instances.lp_powerlaw(7, 3000, 6000, 60000)
    A = engine.Matrix.from_instance(inst)
    rc, r, c = engine.scale_factors(A, engine.SCALE_RUIZ | engine.SCALE_POCK_CHAMBOLLE, 100, 1e-2)
    assert rc == 0
    r1, c1, conv = oracle.ruiz(inst, 100, 1e-2)
    rows = np.repeat(np.arange(inst["m"]), np.diff(inst["ptr"]))
    scaled = dict(inst)
    scaled["val"] = inst["val"] * r1[rows] * c1[inst["idx"]]
    r2, c2 = oracle.pock_chambolle(scaled, 1.0)
    assert np.allclose(r, r1 * r2, rtol=1e-13, atol=0) and np.allclose(c, c1 * c2, rtol=1e-13, atol=0)
