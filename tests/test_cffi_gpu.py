"""The Python cffi binding at run time (lasp-d3_b200/d3_cffi.py, the API of the reference's
src/d3_cffi.py:96-120): D3Calculator.compute() (float in and out, the reference's own
consumer path) against the FP64 oracle at float level, compute_f64() of the same handle at
the FP64 bar, and D3BatchCalculator against per-structure D3Calculator results. The oracle
gets the float-rounded inputs the float ABI sees."""
import numpy as np
import pytest

import d3_systems as S
import oracle

pytestmark = pytest.mark.gpu
cffi = pytest.importorskip("cffi")


def _f32(sys_):
    return {"pos": np.asarray(sys_["pos"], np.float32).astype(np.float64), "Z": sys_["Z"],
            "cell": np.asarray(sys_["cell"], np.float32).astype(np.float64)}


@pytest.mark.parametrize("atm", [None, 40.0])
def test_calculator_matches_oracle(atm):
    import d3_cffi

    s = _f32(S.triclinic_box(300, seed=8))
    calc = d3_cffi.D3Calculator(sorted(set(int(z) for z in s["Z"])), len(s["Z"]), cutoff_radius=95.0,
                                cn_cutoff_radius=40.0, damping_type=1, functional_type=0, atm_cutoff=atm)
    calc.set_cell(s["cell"])
    calc.set_atoms(s["pos"], s["Z"])
    e, f, st = calc.compute()
    assert f.dtype == np.float32 and f.shape == (len(s["Z"]), 3) and st.shape == (3, 3)
    r = oracle.compute(s["pos"], s["Z"], s["cell"], rc=95.0, rc_cn=40.0, rc_atm=atm, damping=1, functional=0)
    assert abs(e - r["energy"]) <= 1e-6 * abs(r["energy"])  # float output of an FP64 evaluation
    assert np.abs(f - r["forces"]).max() <= 1e-6 * np.abs(r["forces"]).max() + 1e-7
    assert np.abs(st - r["stress"]).max() <= 1e-6 * np.abs(r["stress"]).max() + 1e-9
    e64, f64, s64 = calc.compute_f64()
    assert abs(e64 - r["energy"]) <= 1e-9 * abs(r["energy"])
    np.testing.assert_allclose(f64, r["forces"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(s64, r["stress"], rtol=0, atol=1e-7)
    calc.clear()
    del calc


def test_batch_calculator_matches_single_structures():
    import d3_cffi

    structs = [S.triclinic_box(120, seed=2), S.water_box(1), S.triclinic_box(200, seed=4)]
    el = sorted(set(int(z) for s in structs for z in s["Z"]))
    b = d3_cffi.D3BatchCalculator(el, 4, sum(len(s["Z"]) for s in structs), atm_cutoff=40.0)
    b.set_structures([(s["pos"], s["Z"], s["cell"]) for s in structs])
    E, F, ST = b.compute()
    for k, s in enumerate(structs):
        c = d3_cffi.D3Calculator(el, len(s["Z"]), cutoff_radius=95.0, cn_cutoff_radius=40.0, damping_type=1,
                                 functional_type=0, atm_cutoff=40.0)
        c.set_cell(s["cell"])
        c.set_atoms(s["pos"], s["Z"])
        e, f, st = c.compute_f64()
        # the single handle takes float coordinates, the batch doubles: agree at float level
        assert abs(E[k] - e) <= 1e-6 * abs(e)
        assert np.abs(F[k] - f).max() <= 1e-5 * np.abs(f).max()
        assert np.abs(ST[k] - st).max() <= 1e-5 * np.abs(st).max()
