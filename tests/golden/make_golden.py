"""Generate golden vectors from the reference's own CUDA build (oracle/_ref).

Runs on a GPU box (the reference is CUDA-only): for each fixture system it calls the
reference library through its C ABI (init_d3_handle[_with_atm], set_atoms, set_cell,
compute_dispersion_energy_from_handle_status) and stores inputs and float outputs in
tests/golden/reference_outputs.npz. Fixtures: the reference's own property-test
systems (test/d3_test.cpp:343-417) with and without ATM, the 96-atom water box, small
triclinic boxes of the benchmark generator with the 5- and 7-reference tables, and two
low-density boxes on the reference's cell-list path (cubic, and strongly sheared).

    python tests/golden/make_golden.py [out.npz]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "lasp-d3_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import d3_systems as S  # noqa: E402
import ref_lib  # noqa: E402


def perturbed(s, amp, seed):
    rng = np.random.default_rng(seed)
    o = dict(s)
    o["pos"] = s["pos"] + rng.uniform(-amp, amp, s["pos"].shape)
    return o


def fixtures():
    out = []
    small = S.gtest_small_system()
    fe = S.gtest_bcc_fe()
    surf = S.gtest_bcc_fe(True)
    for damping in (0, 1):
        out.append(("small_d%d" % damping, small, dict(rc=40.0, rc_cn=40.0, rc_atm=None, damping=damping, functional=1)))
        out.append(("small_atm_d%d" % damping, small, dict(rc=40.0, rc_cn=40.0, rc_atm=40.0, damping=damping,
                                                          functional=1)))
        out.append(("fe_d%d" % damping, perturbed(fe, 0.1, 0), dict(rc=40.0, rc_cn=40.0, rc_atm=None, damping=damping,
                                                                  functional=1)))
        out.append(("fe_surface_atm_d%d" % damping, perturbed(surf, 0.1, 1),
                    dict(rc=30.0, rc_cn=30.0, rc_atm=30.0, damping=damping, functional=1)))
    out.append(("water_cfg0", S.water_box(0), dict(rc=95.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=0)))
    tric = S.triclinic_box(300, seed=5)
    out.append(("tric300_5ref", tric, dict(rc=60.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=0)))
    out.append(("tric300_7ref", tric, dict(rc=60.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=0, extended=True)))
    # boxes thick enough for the reference's cell-list path (every height above 3 x 95
    # bohr): cubic, and sheared so that its grid cells along x are thinner than the cutoff
    cfg = dict(rc=95.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=0)
    out.append(("celllist_cubic", S.cell_list_box(400, seed=31, edge=160.0), dict(cfg)))
    out.append(("celllist_sheared", S.cell_list_box(500, seed=31, edge=250.0, shear=1.0), dict(cfg)))
    return out


def main(path=None):
    path = path or os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_outputs.npz")
    data = {}
    names = []
    for name, s, kw in fixtures():
        ext = kw.pop("extended", False)
        e, f, st, status = ref_lib.run(s["pos"], s["Z"], s["cell"], extended=ext, **kw)
        names.append(name)
        data[name + "/pos"] = np.asarray(s["pos"], np.float32)
        data[name + "/Z"] = np.asarray(s["Z"], np.uint16)
        data[name + "/cell"] = np.asarray(s["cell"], np.float32)
        data[name + "/params"] = np.array([kw["rc"], kw["rc_cn"], kw["rc_atm"] or 0.0, kw["damping"],
                                           kw["functional"], 1.0 if ext else 0.0])
        data[name + "/energy"] = np.float32(e)
        data[name + "/forces"] = f
        data[name + "/stress"] = st
        data[name + "/status"] = np.int32(status)
        print("%-22s E = %.7f eV  status %d" % (name, e, status))
    data["names"] = np.array(names)
    np.savez(path, **data)
    print("wrote", path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
