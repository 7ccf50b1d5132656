"""Learned ATM surrogate: model file, labelled data, training on the GPU with the
library's own kernels, and use through an engine handle.

The surrogate predicts each atom's share of the Axilrod-Teller-Muto energy (one third of
every triplet through the atom) from per-atom descriptors (include/d3.h documents the
descriptor and the network). Training runs entirely in libd3.so's kernels:
d3_mlp_train_batch (fused BF16 forward/backward + weight-gradient GEMMs) and d3_mlp_adam;
torch only provides device memory, index permutations and the stream.

    import d3_surrogate as SU
    model = SU.Model.load(SU.DEFAULT_MODEL)
    d3 = D3(...); d3.set_surrogate(model)     # ATM now through the surrogate + fallback

Model file (version 1, little-endian):
    b"D3SURR01", uint32 length, JSON header {version, channel_z, members, nparam,
    e_scale, rbf, rc_atm_bohr, meta}, then float32 mean[nf], inv_std[nf], e_shift[nch],
    then per member: W1, W2, W3 as BF16 (uint16, [in][out] row-major), float32
    b1, b2, b3, w4 (128 each) and b4.
"""
import json
import math
import os
import struct
import time

import numpy as np

from d3_b200 import OPT_PRECISION, D3Batch, load_library

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "surrogate", "atm_hcnosicu.d3s")
MAGIC = b"D3SURR01"
NRBF, HID = 32, 128
RBF = {"n": NRBF, "mu0_A": 0.8, "mu1_A": 21.0, "sigma_A": 0.7}
CHANNELS_HCNOSICU = (1, 6, 7, 8, 14, 29)


def layout(nch):
    """Offsets of one member's parameter vector (see d3_mlp_layout)."""
    out = np.zeros(12, np.uint64)
    lib = load_library()
    if lib.d3_mlp_layout(int(nch), out.ctypes.data):
        raise RuntimeError(lib.d3_last_error().decode())
    keys = ("in_dim", "in_pad", "oW1", "ob1", "oW2", "ob2", "oW3", "ob3", "ow4", "ob4", "nparam", "packed")
    return dict(zip(keys, (int(v) for v in out)))


def layout_py(nch):
    """Same offsets without the library (for file I/O on machines without a GPU)."""
    in_dim = nch * NRBF + nch
    in_pad = (in_dim + 15) // 16 * 16
    L = {"in_dim": in_dim, "in_pad": in_pad}
    o = 0
    for name, size in (("oW1", in_pad * HID), ("ob1", HID), ("oW2", HID * HID), ("ob2", HID), ("oW3", HID * HID),
                       ("ob3", HID), ("ow4", HID), ("ob4", 1)):
        L[name] = o
        o += size
    L["nparam"] = (o + 3) // 4 * 4
    return L


def _bf16_bits(x):
    u = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def _from_bf16_bits(b):
    return (np.asarray(b, np.uint32) << 16).view(np.float32)


class Model:
    """Ensemble parameters and normalisation of the surrogate."""

    def __init__(self, channel_z, members, params, mean, inv_std, e_shift, e_scale, meta=None):
        self.channel_z = [int(z) for z in channel_z]
        self.members = int(members)
        self.params = np.ascontiguousarray(params, np.float32).reshape(self.members, -1)
        self.mean = np.ascontiguousarray(mean, np.float32)
        self.inv_std = np.ascontiguousarray(inv_std, np.float32)
        self.e_shift = np.ascontiguousarray(e_shift, np.float32)
        self.e_scale = float(e_scale)
        self.meta = dict(meta or {})
        L = layout_py(len(self.channel_z))
        if self.params.shape[1] != L["nparam"]:
            raise ValueError("parameter vector has %d entries, layout needs %d" % (self.params.shape[1], L["nparam"]))

    @property
    def nch(self):
        return len(self.channel_z)

    def as_dict(self):
        return {"channel_z": self.channel_z, "members": self.members, "params": self.params, "mean": self.mean,
                "inv_std": self.inv_std, "e_shift": self.e_shift, "e_scale": self.e_scale}

    @classmethod
    def init(cls, channel_z, members=4, seed=0):
        """Random initial ensemble (uniform fan-in scaled weights, zero biases)."""
        nch = len(channel_z)
        L = layout_py(nch)
        rng = np.random.default_rng(seed)
        P = np.zeros((members, L["nparam"]), np.float32)
        for m in range(members):
            fan = L["in_dim"]
            b = math.sqrt(6.0 / fan)
            W1 = np.zeros((L["in_pad"], HID), np.float32)
            W1[:fan] = rng.uniform(-b, b, (fan, HID))
            P[m, L["oW1"]:L["ob1"]] = W1.ravel()
            b = math.sqrt(6.0 / HID)
            P[m, L["oW2"]:L["ob2"]] = rng.uniform(-b, b, HID * HID)
            P[m, L["oW3"]:L["ob3"]] = rng.uniform(-b, b, HID * HID)
            P[m, L["ow4"]:L["ob4"]] = rng.uniform(-0.1 * b, 0.1 * b, HID)
        nf = nch * NRBF
        return cls(channel_z, members, P, np.zeros(nf), np.ones(nf), np.zeros(nch), 1.0)

    def save(self, path):
        L = layout_py(self.nch)
        hdr = {"version": 1, "channel_z": self.channel_z, "members": self.members, "nparam": L["nparam"],
               "e_scale": self.e_scale, "rbf": RBF, "rc_atm_bohr": self.meta.get("rc_atm_bohr", 40.0),
               "meta": self.meta}
        hb = json.dumps(hdr, sort_keys=True).encode()
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        with open(path + ".tmp", "wb") as f:
            f.write(MAGIC)
            f.write(struct.pack("<I", len(hb)))
            f.write(hb)
            for a in (self.mean, self.inv_std, self.e_shift):
                f.write(np.asarray(a, "<f4").tobytes())
            for m in range(self.members):
                p = self.params[m]
                for o0, o1 in ((L["oW1"], L["ob1"]), (L["oW2"], L["ob2"]), (L["oW3"], L["ob3"])):
                    f.write(_bf16_bits(p[o0:o1]).astype("<u2").tobytes())
                for o0, o1 in ((L["ob1"], L["oW2"]), (L["ob2"], L["oW3"]), (L["ob3"], L["ow4"]),
                               (L["ow4"], L["ob4"] + 1)):
                    f.write(np.asarray(p[o0:o1], "<f4").tobytes())
        os.replace(path + ".tmp", path)

    @classmethod
    def load(cls, path):
        with open(path, "rb") as f:
            buf = f.read()
        if buf[:8] != MAGIC:
            raise ValueError("%s is not a surrogate model file" % path)
        (hl,) = struct.unpack("<I", buf[8:12])
        hdr = json.loads(buf[12:12 + hl].decode())
        if hdr.get("version") != 1:
            raise ValueError("unsupported surrogate model version %r" % hdr.get("version"))
        nch, M = len(hdr["channel_z"]), int(hdr["members"])
        L = layout_py(nch)
        nf = nch * NRBF
        off = 12 + hl

        def take(dtype, count):
            nonlocal off
            a = np.frombuffer(buf, dtype, count, off)
            off += a.nbytes
            return a

        mean, inv_std, e_shift = take("<f4", nf), take("<f4", nf), take("<f4", nch)
        P = np.zeros((M, L["nparam"]), np.float32)
        for m in range(M):
            for o0, o1 in ((L["oW1"], L["ob1"]), (L["oW2"], L["ob2"]), (L["oW3"], L["ob3"])):
                P[m, o0:o1] = _from_bf16_bits(take("<u2", o1 - o0))
            for o0, o1 in ((L["ob1"], L["oW2"]), (L["ob2"], L["oW3"]), (L["ob3"], L["ow4"]), (L["ow4"], L["ob4"] + 1)):
                P[m, o0:o1] = take("<f4", o1 - o0)
        meta = dict(hdr.get("meta", {}))
        meta["rc_atm_bohr"] = hdr.get("rc_atm_bohr", 40.0)
        return cls(hdr["channel_z"], M, P, mean, inv_std, e_shift, hdr["e_scale"], meta)


# ------------------------------------------------------------------------------------
# labelled data from the exact ATM kernel
# ------------------------------------------------------------------------------------
def label_structures(structs, channel_z=CHANNELS_HCNOSICU, rc_atm=40.0, precision=1, max_batch_atoms=400000,
                     max_batch_structs=2048, log=None):
    """Descriptors and exact per-atom ATM energies (eV) of every atom of `structs`, on the
    device: returns torch tensors G [N, nch*32] float32, center [N] int32, e_atm [N] float64
    and the structure index of each atom [N] int32 (numpy)."""
    import torch

    nch = len(channel_z)
    counts = np.array([len(s["Z"]) for s in structs], np.int64)
    N = int(counts.sum())
    G = torch.empty((N, nch * NRBF), dtype=torch.float32, device="cuda")
    center = torch.empty(N, dtype=torch.int32, device="cuda")
    e_atm = torch.empty(N, dtype=torch.float64, device="cuda")
    sid = np.repeat(np.arange(len(structs), dtype=np.int32), counts)
    stream = torch.cuda.current_stream().cuda_stream
    h = D3Batch(channel_z, max_batch_structs, max_batch_atoms, rc=rc_atm, rc_cn=rc_atm, rc_atm=rc_atm)
    h.set_option(OPT_PRECISION, int(precision))
    s0, a0, t0 = 0, 0, time.time()
    while s0 < len(structs):
        s1, na = s0, 0
        while s1 < len(structs) and s1 - s0 < max_batch_structs and na + counts[s1] <= max_batch_atoms:
            na += counts[s1]
            s1 += 1
        if s1 == s0:
            raise ValueError("structure %d has more atoms than max_batch_atoms" % s0)
        h.set_structures(structs[s0:s1])
        h.compute()
        h.surrogate_descriptors(channel_z, G[a0:].data_ptr(), center[a0:].data_ptr(), e_atm[a0:].data_ptr(), stream)
        s0, a0 = s1, a0 + int(na)
        if log:
            log("labelled %d / %d structures (%d atoms, %.1f s)" % (s0, len(structs), a0, time.time() - t0))
    h.close()
    torch.cuda.synchronize()
    return G, center, e_atm, sid


def descriptors_of(handle, channel_z):
    """Descriptors, centre channels and exact per-atom ATM energies of a computed handle."""
    import torch

    n = handle.n if hasattr(handle, "n") else int(np.sum(handle.counts))
    G = torch.empty((n, len(channel_z) * NRBF), dtype=torch.float32, device="cuda")
    c = torch.empty(n, dtype=torch.int32, device="cuda")
    e = torch.empty(n, dtype=torch.float64, device="cuda")
    handle.surrogate_descriptors(channel_z, G.data_ptr(), c.data_ptr(), e.data_ptr(),
                                 torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return G, c, e


def fit_normalisation(G, center, e_atm, nch, rows, sample=400000, seed=0):
    """Descriptor mean / inverse std and per-channel energy shift / scale from the rows
    `rows` (a subsample of at most `sample` rows is taken to the host)."""
    import torch

    rng = np.random.default_rng(seed)
    sel = rows if len(rows) <= sample else np.sort(rng.choice(rows, sample, replace=False))
    idx = torch.as_tensor(sel, device="cuda", dtype=torch.int64)
    Gs = G.index_select(0, idx).cpu().numpy().astype(np.float64)
    mean = Gs.mean(0)
    std = Gs.std(0)
    inv_std = np.where(std > 1e-12 * (np.abs(mean) + 1.0), 1.0 / np.maximum(std, 1e-30), 1.0)
    c = center.cpu().numpy()[rows]
    y = e_atm.cpu().numpy()[rows]
    shift = np.zeros(nch)
    for k in range(nch):
        if np.any(c == k):
            shift[k] = y[c == k].mean()
    scale = float(np.std(y - shift[c])) or 1.0
    return mean, inv_std, shift, scale


# ------------------------------------------------------------------------------------
# training
# ------------------------------------------------------------------------------------
class Trainer:
    """Adam training of the ensemble on device-resident rows, one launch pair per step
    (d3_mlp_train_batch, d3_mlp_adam). Each member sees its own permutation of the rows."""

    def __init__(self, model, G, center, target, rows, batch=4096, weight_decay=1e-5, seed=0):
        import torch

        self.torch = torch
        self.lib = load_library()
        self.model = model
        self.nch, self.M = model.nch, model.members
        self.L = layout(self.nch)
        if batch % 128:
            raise ValueError("batch must be a multiple of 128")
        self.B = batch
        self.splits = batch // 128
        self.wd = weight_decay
        dev = "cuda"
        self.G, self.center = G, center
        self.target = target.to(dev, torch.float32).contiguous()
        self.rows = torch.as_tensor(np.asarray(rows), device=dev, dtype=torch.int64)
        self.params = torch.as_tensor(model.params.reshape(-1), device=dev).clone()
        self.packed = torch.zeros(self.M * self.L["packed"], dtype=torch.int16, device=dev)
        self.m1 = torch.zeros_like(self.params)
        self.m2 = torch.zeros_like(self.params)
        self.mean = torch.as_tensor(model.mean, device=dev)
        self.inv_std = torch.as_tensor(model.inv_std, device=dev)
        self.acts = torch.empty(self.M * int(self.lib.d3_mlp_acts_elems(self.nch, batch)), dtype=torch.int16,
                                device=dev)
        self.partial = torch.empty(self.M * self.splits * self.L["nparam"], dtype=torch.float32, device=dev)
        self.loss = torch.empty(self.M * self.splits, dtype=torch.float32, device=dev)
        self.E = torch.empty(self.M * batch, dtype=torch.float32, device=dev)
        self.gen = torch.Generator(device=dev)
        self.gen.manual_seed(seed)
        self.step_count = 0
        self._check(self.lib.d3_mlp_pack(self.nch, self.M, self.params.data_ptr(), self.packed.data_ptr(),
                                         self._stream()))

    def _stream(self):
        return self.torch.cuda.current_stream().cuda_stream

    def _check(self, rc):
        if rc:
            raise RuntimeError(self.lib.d3_last_error().decode())

    def step(self, idx, lr):
        """One Adam step on rows idx [members, B] (int32 device tensor); returns the device
        loss buffer (summed squared error per member and split)."""
        torch = self.torch
        s = self._stream()
        self._check(self.lib.d3_mlp_train_batch(self.nch, self.M, self.params.data_ptr(), self.packed.data_ptr(),
                                                self.mean.data_ptr(), self.inv_std.data_ptr(), self.G.data_ptr(),
                                                self.center.data_ptr(), self.target.data_ptr(), idx.data_ptr(),
                                                self.B, self.E.data_ptr(), self.acts.data_ptr(),
                                                self.partial.data_ptr(), self.loss.data_ptr(), s))
        self.step_count += 1
        self._check(self.lib.d3_mlp_adam(self.nch, self.M, self.params.data_ptr(), self.packed.data_ptr(),
                                         self.m1.data_ptr(), self.m2.data_ptr(), self.partial.data_ptr(), self.splits,
                                         float(lr), 0.9, 0.999, 1e-8, float(self.wd), self.step_count, s))
        return self.loss

    def epoch(self, lr_at):
        """One pass over the rows (each member its own permutation); lr_at(step) gives the
        learning rate. Returns the mean training loss per member (normalised units)."""
        torch = self.torch
        nrow = len(self.rows)
        steps = nrow // self.B
        perms = torch.stack([self.rows[torch.randperm(nrow, generator=self.gen, device="cuda")]
                             for _ in range(self.M)]).to(torch.int32)
        acc = torch.zeros(self.M, dtype=torch.float64, device="cuda")
        for k in range(steps):
            idx = perms[:, k * self.B:(k + 1) * self.B].contiguous()
            loss = self.step(idx, lr_at(self.step_count))
            acc += loss.view(self.M, self.splits).sum(1).double()
        return (acc / max(1, steps * self.B)).cpu().numpy()

    def export(self):
        P = self.params.view(self.M, -1).cpu().numpy()
        return Model(self.model.channel_z, self.M, P, self.model.mean, self.model.inv_std, self.model.e_shift,
                     self.model.e_scale, self.model.meta)


def predict(model, G, center, with_grad=False):
    """Ensemble outputs on device rows: per-atom energies [members, n] (eV, including the
    channel shift) and, with_grad, the ensemble-mean dE/dG [n, nch*32] (eV per unit)."""
    import torch

    lib = load_library()
    L = layout(model.nch)
    n = G.shape[0]
    dev = "cuda"
    P = torch.as_tensor(model.params.reshape(-1), device=dev)
    packed = torch.zeros(model.members * L["packed"], dtype=torch.int16, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    if lib.d3_mlp_pack(model.nch, model.members, P.data_ptr(), packed.data_ptr(), s):
        raise RuntimeError(lib.d3_last_error().decode())
    mean = torch.as_tensor(model.mean, device=dev)
    istd = torch.as_tensor(model.inv_std, device=dev)
    E = torch.empty(model.members * n, dtype=torch.float32, device=dev)
    dX = torch.empty((n, model.nch * NRBF), dtype=torch.float32, device=dev) if with_grad else None
    if lib.d3_mlp_forward(model.nch, model.members, P.data_ptr(), packed.data_ptr(), mean.data_ptr(),
                          istd.data_ptr(), G.data_ptr(), center.data_ptr(), n, E.data_ptr(),
                          dX.data_ptr() if with_grad else None, s):
        raise RuntimeError(lib.d3_last_error().decode())
    torch.cuda.synchronize()
    shift = torch.as_tensor(model.e_shift, device=dev).double()[center.long()]
    e = E.view(model.members, n).double() * model.e_scale + shift[None, :]
    if with_grad:
        return e, dX.double() * (model.e_scale / model.members)
    return e


def train(G, center, e_atm, train_rows, val_rows, channel_z=CHANNELS_HCNOSICU, members=4, epochs=40, batch=4096,
          lr=2e-3, lr_min=2e-5, weight_decay=1e-5, seed=0, log=None):
    """Fit normalisation, train the ensemble with a cosine learning-rate schedule and
    return (model, history)."""
    import torch

    nch = len(channel_z)
    mean, inv_std, shift, scale = fit_normalisation(G, center, e_atm, nch, train_rows, seed=seed)
    model = Model.init(channel_z, members, seed=seed)
    model.mean, model.inv_std = mean.astype(np.float32), inv_std.astype(np.float32)
    model.e_shift, model.e_scale = shift.astype(np.float32), scale
    shift_d = torch.as_tensor(shift, device="cuda")
    target = ((e_atm - shift_d[center.long()]) / scale).float()
    tr = Trainer(model, G, center, target, train_rows, batch=batch, weight_decay=weight_decay, seed=seed)
    total = epochs * (len(train_rows) // batch)

    def lr_at(step):
        return lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * min(step, total) / max(total, 1)))

    hist = []
    vidx = torch.as_tensor(np.asarray(val_rows), device="cuda", dtype=torch.int64)
    Gv, cv, yv = G.index_select(0, vidx), center.index_select(0, vidx), e_atm.index_select(0, vidx)
    t0 = time.time()
    for ep in range(epochs):
        loss = tr.epoch(lr_at)
        m = tr.export()
        e = predict(m, Gv, cv)
        err = e.mean(0) - yv
        rec = {"epoch": ep, "train_rmse_ev": (np.sqrt(loss) * scale).tolist(),
               "val_rmse_ev": float(err.pow(2).mean().sqrt()), "val_std_ev": float(e.std(0, unbiased=False).mean()),
               "seconds": time.time() - t0}
        hist.append(rec)
        if log:
            log("epoch %d: train rmse %s meV, val rmse %.4f meV, mean ensemble std %.4f meV (%.1f s)" %
                (ep, " ".join("%.4f" % (1e3 * v) for v in rec["train_rmse_ev"]), 1e3 * rec["val_rmse_ev"],
                 1e3 * rec["val_std_ev"], rec["seconds"]))
    model = tr.export()
    return model, hist
