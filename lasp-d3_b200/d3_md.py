"""MD harness on the graph-captured evaluation.

Two consumers of the D3 path, as in the reference's own drivers:

* ``D3ASECalculator``: the ASE calculator pattern of the reference's example
  (examples/ase_mace_laspd3.py:17-94): energy, forces and Voigt stress of D3 for an
  ``ase.Atoms``; it subclasses ASE's Calculator when ASE is installed and otherwise keeps
  the same ``calculate`` / ``results`` interface.
* ``GraphMD``: one MD step captured once in a CUDA graph and replayed, so a trajectory
  runs with no host round trip per step. ``mode="random-walk"`` is the reference's
  src/test_d3_cffi.py loop (uniform displacement in [-step, step] per coordinate, then
  energy/forces/stress); ``mode="nve"`` is velocity Verlet on the D3 forces.

    python lasp-d3_b200/d3_md.py structure.arc|structure.extxyz STEPS [--mode nve] [--dt 0.5]
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from d3_b200 import D3, OPT_ATM_FORCE_SCALED, OPT_PRECISION  # noqa: E402

# standard atomic weights (amu) of the elements the harness integrates; velocity Verlet
# refuses other elements
MASS = {1: 1.008, 2: 4.0026, 3: 6.94, 4: 9.0122, 5: 10.81, 6: 12.011, 7: 14.007, 8: 15.999, 9: 18.998, 10: 20.180,
        11: 22.990, 12: 24.305, 13: 26.982, 14: 28.085, 15: 30.974, 16: 32.06, 17: 35.45, 18: 39.948, 19: 39.098,
        20: 40.078, 26: 55.845, 27: 58.933, 28: 58.693, 29: 63.546, 30: 65.38, 35: 79.904, 47: 107.87, 53: 126.90,
        78: 195.08, 79: 196.97}
# 1 eV / (A amu) in A / fs^2
ACC_UNIT = 9.648533212e-3
# 1 amu A^2 / fs^2 in eV
KE_UNIT = 103.6426965


class _NoASE:
    """Minimal stand-in for ase's Calculator when ASE is not installed."""

    def __init__(self, **kwargs):
        self.results = {}
        self.atoms = None

    def calculate(self, atoms=None, properties=None, system_changes=None):
        if atoms is not None:
            self.atoms = atoms


try:
    from ase.calculators.calculator import Calculator as _Base
    from ase.calculators.calculator import all_changes as _ALL
except ImportError:  # ASE is optional
    _Base, _ALL = _NoASE, None


class D3ASECalculator(_Base):
    """D3(BJ/zero)(+ATM) for ASE: results energy (eV), forces (eV/A), stress (Voigt,
    eV/A^3, the engine's stress is already divided by the volume)."""

    implemented_properties = ["energy", "forces", "stress"]

    def __init__(self, rc=95.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=0, precision=False, **kwargs):
        super().__init__(**kwargs)
        self.kw = dict(rc=rc, rc_cn=rc_cn, rc_atm=rc_atm, damping=damping, functional=functional)
        self.precision = precision
        self._d3 = None
        self._key = None

    def _handle(self, Z):
        key = tuple(sorted(set(int(z) for z in Z))), len(Z)
        if self._d3 is None or key != self._key:
            self._d3 = D3(Z, len(Z), **self.kw)
            self._d3.set_option(OPT_PRECISION, 1 if self.precision else 0)
            self._key = key
        return self._d3

    def calculate(self, atoms=None, properties=None, system_changes=_ALL):
        if _Base is _NoASE:
            _NoASE.calculate(self, atoms)
        else:
            super().calculate(atoms, properties, system_changes)
        a = self.atoms
        Z = np.asarray(a.get_atomic_numbers())
        d = self._handle(Z)
        d.set_cell(np.asarray(a.get_cell()[:], float))
        d.set_atoms(np.asarray(a.get_positions(), float), Z)
        e, f, s = d.compute()
        self.results["energy"] = e
        self.results["forces"] = f
        self.results["stress"] = np.array([s[0, 0], s[1, 1], s[2, 2], s[1, 2], s[0, 2], s[0, 1]])


class GraphMD:
    """A trajectory of one structure with every step replayed from one CUDA graph."""

    def __init__(self, structure, mode="random-walk", step=0.01, dt=0.5, precision=True, rc=95.0, rc_cn=40.0,
                 rc_atm=40.0, damping=1, functional=0, seed=0, max_steps=100000):
        import torch

        self.torch = torch
        self.mode = mode
        Z = np.asarray(structure["Z"])
        self.n = n = len(Z)
        self.d = D3(Z, n, rc=rc, rc_cn=rc_cn, rc_atm=rc_atm, damping=damping, functional=functional)
        self.d.set_option(OPT_PRECISION, 1 if precision else 0)
        self.d.set_option(OPT_ATM_FORCE_SCALED, 1)  # forces = -dE/dx for the integrator
        self.d.set_cell(structure["cell"])
        self.d.set_atoms(structure["pos"], Z)
        self.d.compute()  # sizes the neighbour lists before the capture
        dev = "cuda"
        self.pos = torch.tensor(np.asarray(structure["pos"], float), dtype=torch.float64, device=dev)
        self.res = torch.zeros(10 + 3 * n, dtype=torch.float64, device=dev)
        self.noise = torch.empty_like(self.pos)
        self.hist = torch.zeros(max_steps, dtype=torch.float64, device=dev)
        self.kin = torch.zeros(max_steps, dtype=torch.float64, device=dev)
        self.k = torch.zeros(1, dtype=torch.int64, device=dev)
        self.step_size, self.dt = float(step), float(dt)
        self.max_steps = max_steps
        torch.cuda.manual_seed(seed)  # the default generator: captured graphs replay its stream
        if mode == "nve":
            try:
                m = np.array([MASS[int(z)] for z in Z])
            except KeyError as ex:
                raise ValueError("velocity Verlet needs the mass of element Z=%s" % ex) from None
            self.minv = torch.tensor(ACC_UNIT / m, dtype=torch.float64, device=dev)[:, None]
            self.mass = torch.tensor(m, dtype=torch.float64, device=dev)[:, None]
            self.vel = torch.zeros_like(self.pos)
            self._evaluate(torch.cuda.current_stream())
            torch.cuda.synchronize()
            self.acc = self.res[1:1 + 3 * n].view(n, 3) * self.minv
        self.stream = torch.cuda.Stream()
        self.stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(self.stream):
            self._step()  # warm-up outside the capture
        torch.cuda.synchronize()
        self.k.zero_()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=self.stream):
            self._step()
        torch.cuda.synchronize()

    def _evaluate(self, stream):
        s = stream.cuda_stream
        self.d.set_positions_device(self.pos.data_ptr(), s)
        self.d.compute_async(s)
        self.d.copy_results_device(self.res.data_ptr(), s)

    def _step(self):
        torch = self.torch
        s = torch.cuda.current_stream()
        n = self.n
        if self.mode == "random-walk":
            self.noise.uniform_(-self.step_size, self.step_size)
            self.pos.add_(self.noise)
            self._evaluate(s)
        else:
            dt = self.dt
            self.pos.add_(self.vel * dt + 0.5 * self.acc * (dt * dt))
            self._evaluate(s)
            acc_new = self.res[1:1 + 3 * n].view(n, 3) * self.minv
            self.vel.add_(0.5 * (self.acc + acc_new) * dt)
            self.acc.copy_(acc_new)
            self.kin.index_copy_(0, self.k, (0.5 * KE_UNIT * (self.mass * self.vel * self.vel).sum()).view(1))
        self.hist.index_copy_(0, self.k, self.res[0:1])
        self.k.add_(1)

    def set_velocities(self, v):
        """Initial velocities (A/fs) for mode="nve"."""
        self.vel.copy_(self.torch.as_tensor(v, dtype=self.torch.float64))

    def run(self, steps):
        """Replay `steps` steps; returns (potential energies (eV), kinetic energies (eV),
        device seconds)."""
        torch = self.torch
        if int(self.k.item()) + steps > self.max_steps:
            raise ValueError("more steps than max_steps")
        k0 = int(self.k.item())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(self.stream):
            a.record()
            for _ in range(steps):
                self.graph.replay()
            b.record()
        b.synchronize()
        return (self.hist[k0:k0 + steps].cpu().numpy(), self.kin[k0:k0 + steps].cpu().numpy(),
                a.elapsed_time(b) * 1e-3)

    def close(self):
        del self.graph
        self.d.close()


def main():
    import d3_io

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("structure")
    ap.add_argument("steps", type=int)
    ap.add_argument("--mode", choices=["random-walk", "nve"], default="random-walk")
    ap.add_argument("--step", type=float, default=0.01, help="random-walk displacement bound (A)")
    ap.add_argument("--dt", type=float, default=0.5, help="velocity-Verlet time step (fs)")
    ap.add_argument("--fp64", action="store_true", help="FP64 plain form instead of the precision form")
    ap.add_argument("--no-atm", action="store_true")
    a = ap.parse_args()
    s = d3_io.read_structures(a.structure)[0]
    md = GraphMD(s, mode=a.mode, step=a.step, dt=a.dt, precision=not a.fp64, rc_atm=None if a.no_atm else 40.0,
                 max_steps=max(a.steps, 1))
    t0 = time.time()
    e, k, dev_s = md.run(a.steps)
    wall = time.time() - t0
    print("Running %d steps of %s MD for %d atoms" % (a.steps, a.mode, md.n))
    for i in range(0, a.steps, max(1, a.steps // 10)):
        print("Step %d/%d, Energy: %.6f%s" % (i + 1, a.steps, e[i], "" if a.mode != "nve" else ", Total: %.6f" %
                                                 (e[i] + k[i])))
    print("Average energy: %.6f  std: %.6f" % (e.mean(), e.std()))
    print("Steps per second: %.2f (device), %.2f (wall)" % (a.steps / dev_s, a.steps / wall))
    md.close()


if __name__ == "__main__":
    main()
