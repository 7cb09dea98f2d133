"""Learned absorbing boundary: face-frame features, training pairs recorded
from wide-NPML runs of the method itself, and the GPU trainer.

The solver side (include/nexd.h, nexd_set_boundary_mlp) predicts the exterior
state q+ of every absorbing face from its interior trace q-.  Training pairs
come from a wide model whose NPML starts where the small model's absorbing
faces are: those faces are interior faces of the wide mesh, and the wide run
records both of their traces every step (nexd_get_face_traces).  Features and
targets use the small model's face frames (the tetrahedra are identical), so
x = features(q-) (incoming, outgoing and in-plane values per face node),
y = the incoming values of q+, both divided by the RMS of x.

The network is trained with the library's own forward/backward/Adam kernels
(nexd_mlp_loss_grad, nexd_mlp_adam) on device tensors owned by torch.
"""
import ctypes as C
import os

import numpy as np

from . import _abi, synth

HIDDEN = 128


# ---------------------------------------------------------------------------
# face frames and features (the same arithmetic as the device ghost kernel)
# ---------------------------------------------------------------------------

def face_frames(mesh, elem, face):
    """Outward normal, tangents and the impedances rho*vp, rho*vs of faces (1-based elem, face)."""
    e, f = np.asarray(elem) - 1, np.asarray(face) - 1
    n = mesh.array("nnormal")[:, f, e].T
    s = mesh.array("stangential")[:, f, e].T
    t = mesh.array("ttangential")[:, f, e].T
    rho = mesh.array("rho")[e]
    return n, s, t, rho * mesh.array("vpu")[e], rho * mesh.array("vsu")[e]


def characteristics(q, n, s, t, zp, zs):
    """q (nf, 9, NpF) -> (nf, 9 NpF), node-major (index 9 * node + component):
    per node (w_P, w_S1, w_S2, u_P, u_S1, u_S2, s.S.s, t.S.t, s.S.t) / Zp with
    w = traction - Z velocity (incoming), u = traction + Z velocity (outgoing),
    Z = Zp normal, Zs tangential."""
    nf, _, npf = q.shape
    v = q[:, 6:9, :]
    S = np.empty((nf, 3, 3, npf), dtype=np.float64)
    S[:, 0, 0], S[:, 1, 1], S[:, 2, 2] = q[:, 0], q[:, 1], q[:, 2]
    S[:, 0, 1] = S[:, 1, 0] = q[:, 3]
    S[:, 1, 2] = S[:, 2, 1] = q[:, 4]
    S[:, 0, 2] = S[:, 2, 0] = q[:, 5]
    def proj(a, b):
        return np.einsum("fi,fijk,fj->fk", a, S, b)
    def vel(a):
        return np.einsum("fik,fi->fk", v, a)
    zp_, ks = zp[:, None], (zs / zp)[:, None]
    snn, sns, snt = proj(n, n) / zp_, proj(n, s) / zp_, proj(n, t) / zp_
    vn, vs, vt = vel(n), vel(s), vel(t)
    x = np.stack([snn - vn, sns - ks * vs, snt - ks * vt, snn + vn, sns + ks * vs, snt + ks * vt,
                  proj(s, s) / zp_, proj(t, t) / zp_, proj(s, t) / zp_], axis=1)  # (nf, 9, NpF)
    return np.ascontiguousarray(x.transpose(0, 2, 1).reshape(nf, 9 * npf))


def features(q, n, s, t, zp, zs):
    """Network input of face traces q (the device ghost kernel's features):
    the characteristics with the trace's own incoming values w set to zero."""
    x = characteristics(q, n, s, t, zp, zs)
    nf = x.shape[0]
    x.reshape(nf, -1, 9)[..., :3] = 0.0
    return x


def incoming_only(y, npf):
    """Targets: the incoming values w of each node, the other six components zero."""
    nf = y.shape[0]
    out = np.zeros_like(y).reshape(nf, npf, 9)
    out[..., :3] = y.reshape(nf, npf, 9)[..., :3]
    return out.reshape(nf, 9 * npf)


def ghost_states(xn, yn, r, n, s, t, zp, rho_max, npf):
    """The exterior states the solver uses (the arithmetic of the device ghost
    kernel): the predicted incoming values w, clamped to rho_max times the
    trace's outgoing values u, as the traction w_P n + w_S1 s + w_S2 t with
    zero velocity.  xn, yn (nf, 9 NpF) in RMS units, r the RMS scales."""
    nf = xn.shape[0]
    x = xn.reshape(nf, npf, 9)
    y = yn.reshape(nf, npf, 9)
    b = rho_max * np.abs(x[..., 3:6])
    w = np.clip(y[..., :3], -b, b) * (r * zp)[:, None, None]
    q = np.zeros((nf, 9, npf))
    def comp(i, j):
        return (w[..., 0] * n[:, i, None] * n[:, j, None] +
                w[..., 1] * (n[:, i, None] * s[:, j, None] + s[:, i, None] * n[:, j, None]) +
                w[..., 2] * (n[:, i, None] * t[:, j, None] + t[:, i, None] * n[:, j, None]))
    for c, (i, j) in enumerate(((0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2))):
        q[:, c] = comp(i, j)
    return q


def normalise(x, y=None):
    """Divide by the RMS of x per face (zero faces stay zero)."""
    r = np.sqrt((x.astype(np.float64) ** 2).mean(axis=1))
    inv = np.where(r > 0, 1.0 / np.where(r > 0, r, 1.0), 0.0)[:, None]
    return (x * inv, None if y is None else y * inv, r)


def init_params(nin, hidden=HIDDEN, seed=0):
    """Glorot-uniform W1, W2; zero W3, b3 (the plain absorbing boundary)."""
    rng = np.random.default_rng(seed)
    def glorot(o, i):
        lim = np.sqrt(6.0 / (o + i))
        return rng.uniform(-lim, lim, size=(o, i))
    parts = [glorot(hidden, nin), np.zeros(hidden), glorot(hidden, hidden), np.zeros(hidden),
             np.zeros((nin, hidden)), np.zeros(nin)]
    return np.concatenate([p.ravel() for p in parts]).astype(np.float32)


# ---------------------------------------------------------------------------
# wide / small model pair
# ---------------------------------------------------------------------------

def _default_layers(Lz):
    return [(Lz - 600.0, 3000.0, 1730.0, 2400.0, 9000.0, 9000.0), (-np.inf, 5000.0, 2890.0, 2800.0, 9000.0, 9000.0)]


def write_npml_model(directory, *, cells, h, pml_cells, nt, sources=(), stations=(), layers=None):
    """The small model's box surrounded by pml_cells of NPML on the sides and
    the bottom (free top), with the same undistorted tetrahedra inside.
    Returns the element index (0-based) of every small-model element in it."""
    nx, ny, nz = cells
    P = pml_cells
    Lx, Ly, Lz = nx * h, ny * h, nz * h
    layers = layers or _default_layers(Lz)
    par = dict(timeint=4, nt=nt, cfl=0.3, set_pml=".true.", pml_delta=P * h, pml_rc=0.001, pml_kmax=1.0,
               pml_afac=1.0)
    W = (nx + 2 * P, ny + 2 * P, nz + P)
    synth.write_simulation(directory, box=(-P * h, Lx + P * h, -P * h, Ly + P * h, -P * h, Lz), cells=W, jitter=0.0,
                           layers=layers, pml_cells=P, parfile=par, sources=sources, stations=stations)
    hex_small = np.arange(nx * ny * nz)
    i, j, k = hex_small % nx, (hex_small // nx) % ny, hex_small // (nx * ny)
    hex_wide = (i + P) + W[0] * ((j + P) + W[1] * (k + P))
    return (hex_wide[:, None] * 6 + np.arange(6)[None, :]).ravel()


def write_model_pair(wide_dir, small_dir, *, cells=(8, 8, 4), h=250.0, pml_cells=8, nt=300, sources=(),
                     stations=(), layers=None, f0=3.0):
    """Small model (cells, absorbing sides and bottom, free top) and the wide
    model around it (pml_cells of NPML on the sides and the bottom), with the
    same undistorted tetrahedra inside.  Returns wide element index (0-based)
    of every small element."""
    Lz = cells[2] * h
    layers = layers or _default_layers(Lz)
    par = dict(timeint=4, nt=nt, cfl=0.3)
    synth.write_simulation(small_dir, box=(0.0, cells[0] * h, 0.0, cells[1] * h, 0.0, Lz), cells=cells, jitter=0.0,
                           layers=layers, parfile=par, sources=sources, stations=stations)
    return write_npml_model(wide_dir, cells=cells, h=h, pml_cells=pml_cells, nt=nt, sources=sources,
                            stations=stations, layers=layers)


def record_pairs(wide_solver, wide_elem, face, steps, npf, every=1):
    """Runs the wide model step by step and returns the traces of the given
    faces (1-based wide elements) every `every` steps: (samples, 2, 9, NpF)."""
    out = []
    for it in range(1, steps + 1):
        wide_solver.run(it, it)
        if it % every == 0:
            out.append(wide_solver.face_traces(wide_elem, face, npf)[0])
    return np.concatenate(out, axis=0)


# ---------------------------------------------------------------------------
# training with the library's kernels
# ---------------------------------------------------------------------------

class Trainer:
    """Adam on the MSE of normalised exterior states, on the GPU."""

    def __init__(self, nin, params=None, hidden=HIDDEN, batch=4096, lr=1e-3, seed=0, group=None):
        """group: a replicas.Group for data-parallel training (each rank fits
        its own samples; gradients are averaged over the ranks before every
        Adam step, so all ranks keep the same parameters); None: one process."""
        import torch
        self.torch = torch
        self.group = group
        self.nin, self.hidden, self.batch, self.lr = nin, hidden, batch, lr
        lib = _abi.gpu_lib()
        self.lib = lib
        self.count = lib.nexd_mlp_param_count(nin, hidden)
        p0 = init_params(nin, hidden, seed) if params is None else np.asarray(params, dtype=np.float32)
        assert p0.size == self.count
        dev = torch.device("cuda")
        self.params = torch.from_numpy(p0.copy()).to(dev)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.work = torch.zeros(lib.nexd_mlp_workspace_floats(nin, hidden, batch), dtype=torch.float32, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)
        self.step = 0

    def _ptr(self, t):
        return C.c_void_p(t.data_ptr())

    def loss_grad(self, x, y):
        """Loss and gradient of a device batch (rows <= batch)."""
        st = self.lib.nexd_mlp_loss_grad(self.nin, self.hidden, self._ptr(self.params), self._ptr(x), self._ptr(y),
                                         x.shape[0], self._ptr(self.grads), self._ptr(self.loss), self._ptr(self.work),
                                         None)
        if st != 0:
            raise RuntimeError(f"nexd_mlp_loss_grad failed: {st}")

    def fit(self, x, y, epochs=10, seed=0):
        """x, y: numpy (samples, nin) normalised; returns the loss per epoch."""
        torch = self.torch
        xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()
        yd = torch.from_numpy(np.ascontiguousarray(y, dtype=np.float32)).cuda()
        n = xd.shape[0]
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        hist = []
        from . import replicas
        nbatch = n // self.batch
        if self.group is not None:
            nbatch = replicas.agree_min(self.group, nbatch)  # the same number of all-reduces on every rank
        for _ in range(epochs):
            perm = torch.randperm(n, device="cuda", generator=g)
            tot = torch.zeros((), device="cuda")
            nb = 0
            for bi in range(nbatch):
                idx = perm[bi * self.batch:(bi + 1) * self.batch]
                xb, yb = xd[idx].contiguous(), yd[idx].contiguous()
                self.loss_grad(xb, yb)
                if self.group is not None:
                    replicas.allreduce_mean(self.group, self.grads)
                self.step += 1
                st = self.lib.nexd_mlp_adam(self.count, self._ptr(self.params), self._ptr(self.grads),
                                            self._ptr(self.m), self._ptr(self.v), self.step, self.lr, 0.9, 0.999,
                                            1e-8, None)
                if st != 0:
                    raise RuntimeError(f"nexd_mlp_adam failed: {st}")
                tot += self.loss[0]
                nb += 1
            hist.append(float(tot) / max(nb, 1))
        return hist

    def evaluate(self, x, y):
        """Mean loss over full batches of (x, y)."""
        torch = self.torch
        xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()
        yd = torch.from_numpy(np.ascontiguousarray(y, dtype=np.float32)).cuda()
        tot, nb = 0.0, 0
        for b0 in range(0, xd.shape[0] - self.batch + 1, self.batch):
            self.loss_grad(xd[b0:b0 + self.batch].contiguous(), yd[b0:b0 + self.batch].contiguous())
            tot += float(self.loss[0])
            nb += 1
        return tot / max(nb, 1)

    def parameters(self):
        return self.params.cpu().numpy()


# ---------------------------------------------------------------------------
# end-to-end: training data, training, evaluation against the wide model
# ---------------------------------------------------------------------------

def random_sources(n, cells, h, seed, depth=(300.0, 700.0), f0=3.0, margin=2):
    """Seeded double couples inside the small box (away from its boundary)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = cells
    Lx, Ly, Lz = nx * h, ny * h, nz * h
    out = []
    for _ in range(n):
        strike, dip, rake = rng.uniform(0, 360), rng.uniform(10, 90), rng.uniform(-180, 180)
        x = rng.uniform(margin * h, Lx - margin * h)
        y = rng.uniform(margin * h, Ly - margin * h)
        d = rng.uniform(*depth)
        out.append(dict(xyz=(float(x), float(y), float(Lz - d)), type=1, stf=2, f0=f0,
                        M=synth.double_couple(strike, dip, rake, m0=1e15)))
    return out


def random_layers(n, cells, h, seed, vp=(2500.0, 5500.0), vpvs=(1.6, 1.9), rho=(2200.0, 2900.0)):
    """n seeded two-layer materials (an upper layer 600 m thick over a
    half-space), each layer's vp, vp/vs and density uniform in the given
    ranges; elastic (Q 9000)."""
    rng = np.random.default_rng(seed)
    Lz = cells[2] * h
    out = []
    for _ in range(n):
        lay = []
        for zmin in (Lz - 600.0, -np.inf):
            p = rng.uniform(*vp)
            lay.append((zmin, float(p), float(p / rng.uniform(*vpvs)), float(rng.uniform(*rho)), 9000.0, 9000.0))
        out.append(lay)
    return out


def surface_stations(cells, h, n=9):
    nx, ny, nz = cells
    Lx, Ly, Lz = nx * h, ny * h, nz * h
    g = int(round(np.sqrt(n)))
    xs = np.linspace(0.2 * Lx, 0.8 * Lx, g)
    ys = np.linspace(0.2 * Ly, 0.8 * Ly, g)
    return [(float(x), float(y), Lz) for y in ys for x in xs]


class ModelPair:
    """A small (absorbing) model and its wide-NPML extension for one source;
    with npml_cells, also the small model inside a thin NPML of that many
    elements (the layer the learned boundary is meant to replace)."""

    def __init__(self, root, name, source, *, cells, h, pml_cells, duration, N=4, layers=None, npml_cells=0):
        from .host import Mesh
        self.wide_dir = os.path.join(root, f"{name}_wide")
        self.small_dir = os.path.join(root, f"{name}_small")
        st = surface_stations(cells, h)
        # nt from the small model's dt (same tetrahedra, same dt)
        self.map = write_model_pair(self.wide_dir, self.small_dir, cells=cells, h=h, pml_cells=pml_cells, nt=10,
                                    sources=[source], stations=st, layers=layers)
        probe = Mesh(self.small_dir, N=N, stf_stage_time=True)
        nt = int(np.ceil(duration / probe.dt))
        probe.close()
        self.map = write_model_pair(self.wide_dir, self.small_dir, cells=cells, h=h, pml_cells=pml_cells, nt=nt,
                                    sources=[source], stations=st, layers=layers)
        self.small = Mesh(self.small_dir, N=N, stf_stage_time=True)
        self.wide = Mesh(self.wide_dir, N=N, stf_stage_time=True)
        self.nt = nt
        self.npml = None
        if npml_cells:
            self.npml_dir = os.path.join(root, f"{name}_npml{npml_cells}")
            self.npml_map = write_npml_model(self.npml_dir, cells=cells, h=h, pml_cells=npml_cells, nt=nt,
                                             sources=[source], stations=st, layers=layers)
            self.npml = Mesh(self.npml_dir, N=N, stf_stage_time=True)
        # kinetic-energy weights of the small model: 1/2 rho J M (M the reference mass matrix)
        self._mass = np.linalg.inv(self.small.array("invmass"))
        self._rhoj = 0.5 * self.small.array("rho") * np.abs(self.small.array("jacobian"))
        face = self.small.array("face")
        e, f = np.nonzero(face.T == -2)
        self.bf_small_elem, self.bf_face = e + 1, f + 1
        self.bf_wide_elem = self.map[e] + 1
        self.frames = face_frames(self.small, self.bf_small_elem, self.bf_face)

    def training_pairs(self, Solver, every=2, quiet=1e-3):
        """Normalised (x, y) of the small model's absorbing faces from the wide run."""
        s = Solver(self.wide.desc_ptr)
        tr = record_pairs(s, self.bf_wide_elem, self.bf_face, self.nt, self.small.NpF, every)
        s.close()
        nfc = len(self.bf_face)
        nt_rec = tr.shape[0] // nfc
        n, s_, t, zp, zs = (np.tile(a, (nt_rec, 1)) if a.ndim == 2 else np.tile(a, nt_rec) for a in self.frames)
        x = features(tr[:, 0].astype(np.float64), n, s_, t, zp, zs)
        y = incoming_only(characteristics(tr[:, 1].astype(np.float64), n, s_, t, zp, zs), self.small.NpF)
        xn, yn, r = normalise(x, y)
        keep = r > quiet * r.max()
        return xn[keep].astype(np.float32), yn[keep].astype(np.float32)

    def field_on_small(self, wide_field, emap=None):
        Np = self.small.Np
        emap = self.map if emap is None else emap
        idx = (emap[:, None] * Np + np.arange(Np)[None, :]).ravel()
        return wide_field[idx]

    def kinetic_energy(self, v):
        """Kinetic energy of a velocity field on the small model's nodes,
        v (K Np, 3): sum over elements of 1/2 rho J v_c^T M v_c."""
        Np = self.small.Np
        ve = v.reshape(-1, Np, 3)
        return float(np.einsum("e,enc,nm,emc->", self._rhoj, ve, self._mass, ve))

    def evaluate(self, Solver, params, checkpoints, max_reflection=0.5):
        """Every boundary against the wide NPML run (the reference solution) in
        the small domain: the plain absorbing faces, the learned boundary and,
        when the pair has one, the thin NPML.  Per boundary: the relative L2 of
        the velocity field at the checkpoint steps, the trace misfit of the
        surface stations, and the reflection energy -- the kinetic energy of
        the difference from the reference inside the small domain (inside it
        every model solves the same equations, so the difference is what its
        boundary sent back), as a fraction of the largest kinetic energy of the
        reference in the small domain at the checkpoints."""
        runs = {}
        cases = [("wide", None), ("plain", None), ("learned", params)]
        if self.npml is not None:
            cases.append(("npml", None))
        for label, p in cases:
            mesh = {"wide": self.wide, "npml": self.npml}.get(label, self.small)
            emap = {"wide": self.map, "npml": getattr(self, "npml_map", None)}.get(label)
            s = Solver(mesh.desc_ptr)
            if label == "learned":
                s.set_boundary_mlp(p, max_reflection)
            fields, it0 = [], 1
            for cp in checkpoints:
                s.run(it0, cp)
                it0 = cp + 1
                f = s.field()[:, 6:9].astype(np.float64)
                fields.append(self.field_on_small(f, emap) if emap is not None else f)
            if it0 <= self.nt:
                s.run(it0, self.nt)
            runs[label] = (fields, s.traces()[..., 0].astype(np.float64))
            s.close()
        out = {}
        wf, wt = runs["wide"]
        e_ref = max(self.kinetic_energy(b) for b in wf)
        for label, _ in cases[1:]:
            f, t = runs[label]
            out[label] = {
                "field_err": [float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(f, wf)],
                "trace_err": float(np.linalg.norm(t[:, :, 3:6] - wt[:, :, 3:6]) / np.linalg.norm(wt[:, :, 3:6])),
                "reflection_energy": [self.kinetic_energy(a - b) / e_ref for a, b in zip(f, wf)],
            }
        return out
