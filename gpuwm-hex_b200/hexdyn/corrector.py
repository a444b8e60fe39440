"""Learned corrector: a cheap reduced step plus per-column and per-edge
BF16 tensor-core networks, with the full step as fallback.

The reduced step runs the same dycore either with a time step ``ratio``
times longer and ``ratio`` times as many acoustic substeps (the acoustic
step and its stability unchanged, the large-step tendencies, recovery and
transport done once instead of ``ratio`` times), or with fewer acoustic
substeps at the same time step (``ratio`` 1).  It stands for ``ratio``
full steps.  After it, a column
network (inputs theta_m, rho_zz, w, qv, the cell mean of edge u and the
neighbour mean of theta_m over the levels; 3 hidden layers; outputs the
increments of theta_m, rho_zz and w) and an edge network (inputs u, theta_m
of both cells and their mean rho_zz; outputs the increment of u) correct
the state towards what the ``ratio`` full steps would have produced.  The networks
are trained on pairs of full and reduced steps taken from the same state
(:func:`make_pairs`), entirely with the library's kernels (hexdyn.mlp).

Every corrected step is checked: if the reduced step set its validation
flag, if the total energy (internal + potential + kinetic) changes by more
than ``energy_tol`` relative to the state before the step, or if the RMS of
w grows by more than ``w_growth_tol`` in the step (the signature of an
acoustic instability of the reduced step, which the global energy sees only
late), the step is redone with the full step from the saved state.
"""

from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib, mlp
from .driver import DeviceAtmosphere, HexDycoreDriver

FIELDS = tuple(_lib.FIELDS)


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(int(t.data_ptr()))


def copy_state(dst: HexDycoreDriver, src: HexDycoreDriver) -> None:
    """Device copy of the current state and saved diagnostics (same mesh)."""
    a, b = DeviceAtmosphere(dst), DeviceAtmosphere(src)
    for name in FIELDS:
        if name == "scalars" and src.sizes["n_scalars"] == 0:
            continue
        a.padded(name).copy_(b.padded(name))


def snapshot(drv: HexDycoreDriver) -> dict:
    atm = DeviceAtmosphere(drv)
    return {n: atm.padded(n).clone() for n in FIELDS if not (n == "scalars" and drv.sizes["n_scalars"] == 0)}


def snapshot_into(drv: HexDycoreDriver, snap: dict | None) -> dict:
    """Snapshot into the buffers of an earlier snapshot of the same driver."""
    if snap is None:
        return snapshot(drv)
    atm = DeviceAtmosphere(drv)
    for n, t in snap.items():
        t.copy_(atm.padded(n))
    return snap


def restore(drv: HexDycoreDriver, snap: dict) -> None:
    atm = DeviceAtmosphere(drv)
    for n, t in snap.items():
        atm.padded(n).copy_(t)


class StateFeatures:
    """Device buffers of the raw column and edge features of one mesh."""

    def __init__(self, drv: HexDycoreDriver):
        import torch

        s = drv.sizes
        self.L, self.C, self.E = s["n_levels"], s["n_cells"], s["n_edges"]
        self.col = torch.empty(self.C, 6 * self.L, dtype=torch.float32, device="cuda")
        self.edge = torch.empty(self.E, 4 * self.L, dtype=torch.float32, device="cuda")

    def compute(self, drv: HexDycoreDriver) -> None:
        lib = _lib.load()
        st = drv._stream_handle()
        _lib.check(lib.hexdyn_column_features(drv._handle, _ptr(self.col), self.col.shape[1], st))
        _lib.check(lib.hexdyn_edge_features(drv._handle, _ptr(self.edge), self.edge.shape[1], st))


@dataclass
class Pairs:
    """Training samples: raw features and target increments (full - reduced)."""

    col_x: np.ndarray
    col_y: np.ndarray
    edge_x: np.ndarray
    edge_y: np.ndarray
    pairs: int = 0
    seconds: float = 0.0


def make_pairs(full: HexDycoreDriver, reduced: HexDycoreDriver, states, *, samples: int, steps_between: int = 2,
               times: int = 2, seed: int = 0, ratio: int = 1) -> Pairs:
    """From each initial state (``(state, saved_diagnostics or None)``),
    advance the full driver and, ``times`` times, take ``ratio`` full steps
    and one reduced step from the same state; sample ``samples`` columns
    and edges in total.  Features are those of the reduced result, targets
    the difference full - reduced of theta_m, rho_zz, w (columns) and u
    (edges)."""
    import torch

    t0 = time.perf_counter()
    rng = np.random.default_rng(seed)
    n_pairs = len(states) * times
    per = -(-samples // n_pairs)
    f_full, f_red = StateFeatures(full), StateFeatures(reduced)
    L = f_full.L
    cx, cy, ex, ey = [], [], [], []
    for state, side in states:
        full.set_state(state, side)
        for _ in range(times):
            full.step_async(steps_between)
            copy_state(reduced, full)
            reduced.step_async(1)
            full.step_async(ratio)
            f_full.compute(full)
            f_red.compute(reduced)
            full.synchronize()
            cols = rng.choice(f_full.C, size=min(per, f_full.C), replace=False)
            edges = rng.choice(f_full.E, size=min(per, f_full.E), replace=False)
            ci = torch.from_numpy(cols).cuda()
            ei = torch.from_numpy(edges).cuda()
            xr = f_red.col.index_select(0, ci).cpu().numpy()
            xf = f_full.col.index_select(0, ci).cpu().numpy()
            er = f_red.edge.index_select(0, ei).cpu().numpy()
            ef = f_full.edge.index_select(0, ei).cpu().numpy()
            cx.append(xr)
            cy.append(xf[:, :3 * L] - xr[:, :3 * L])
            ex.append(er)
            ey.append(ef[:, :L] - er[:, :L])
    full.read_flag()
    reduced.read_flag()
    out = Pairs(np.concatenate(cx)[:samples], np.concatenate(cy)[:samples], np.concatenate(ex)[:samples],
                np.concatenate(ey)[:samples], pairs=n_pairs)
    out.seconds = time.perf_counter() - t0
    return out


def rank_batches(n_batches: int, rank: int, world: int) -> list[int]:
    """Data-parallel shard of an epoch's batches: rank r takes batches
    r, r + W, ... and every rank takes the same count (the remainder is
    dropped), so all ranks join the same number of gradient reductions."""
    per_rank = n_batches // world
    return [rank + i * world for i in range(per_rank)]


def average_gradients(tensors, group=None) -> None:
    """Sum every tensor over the ranks of ``group`` and divide by the rank
    count, in place (one all-reduce per tensor, in list order on every rank).
    Each rank's gradient is the mean over its own batch, so the average is
    the mean over the global batch."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        t.div_(world)


def global_mean_loss(loss_sum: float, count: int, group=None) -> float:
    """An epoch's mean training loss over every rank of ``group`` (the
    summed squared errors and the element counts are all-reduced together),
    so every rank records the loss of the global batch sequence; without a
    group, the local mean."""
    if group is None:
        return loss_sum / max(count, 1)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([loss_sum, float(count)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t[0].item()) / max(float(t[1].item()), 1.0)


def _stats(x: np.ndarray, floor: float = 1e-12):
    mean = x.mean(axis=0).astype(np.float32)
    std = x.std(axis=0).astype(np.float32)
    inv = np.where(std > floor, 1.0 / np.maximum(std, floor), 0.0).astype(np.float32)
    return mean, std, inv


@dataclass
class NetTraining:
    train_loss: list = field(default_factory=list)
    val_loss: float = float("nan")
    val_loss_initial: float = float("nan")
    val_loss_zero: float = float("nan")  # normalised loss of applying no correction (zero increments)
    seconds: float = 0.0
    steps: int = 0


class TrainedNet:
    """A TensorCoreMLP with its input normalisation and output scaling."""

    def __init__(self, n_in: int, hidden: int, depth: int, n_out: int, *, seed: int):
        self.net = mlp.TensorCoreMLP(n_in, hidden, depth, n_out, seed=seed)
        self.n_in, self.n_out = n_in, n_out

    def fit(self, x: np.ndarray, y: np.ndarray, *, epochs: int, batch: int, lr: float, val_frac: float = 0.2,
            seed: int = 0, group=None) -> NetTraining:
        """Adam on the mean squared error of normalised targets.  Given a
        process group of W > 1 ranks (``group=torch.distributed.group.WORLD``
        for all of them; every rank given the same pairs and seed, hence the
        same split and initial weights) each rank runs its shard of every
        epoch's batches and the weight and bias gradients are averaged over
        the ranks before each optimizer step, so the weights stay identical
        on every rank (data parallel).  Each epoch runs
        ``(n_batches // W) * W`` batches, so with W > 1 up to W - 1 full
        batches of a reshuffled epoch are left out (a different set each
        epoch); ``train_loss`` is the mean over all ranks' batches.  Without a
        group the rank trains alone."""
        import torch
        import torch.distributed as dist

        world, rank = 1, 0
        if group is not None:
            world, rank = dist.get_world_size(group), dist.get_rank(group)

        rng = np.random.default_rng(seed)
        perm = rng.permutation(len(x))
        n_val = int(round(val_frac * len(x)))
        val, tr = perm[:n_val], perm[n_val:]
        self.x_mean, _, self.x_inv = _stats(x[tr])
        self.y_mean, y_std, _ = _stats(y[tr])
        self.y_scale = np.where(y_std > 0, y_std, 1.0).astype(np.float32)
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
        self.d_x_mean, self.d_x_inv = dev(self.x_mean), dev(self.x_inv)
        self.d_y_scale, self.d_y_shift = dev(self.y_scale), dev(self.y_mean)
        net = self.net
        lib = mlp.load()
        st = mlp._stream()
        yn = ((y - self.y_mean) / self.y_scale).astype(np.float32)
        B = mlp.round_up(batch, 128)
        Xb = torch.empty(B, net.p_in, dtype=torch.bfloat16, device="cuda")
        Xt = torch.empty(net.p_in, B, dtype=torch.bfloat16, device="cuda")
        Tb = torch.zeros(B, net.p_out, dtype=torch.float32, device="cuda")
        raw = torch.empty(B, x.shape[1], dtype=torch.float32, device="cuda")

        def load_batch(idx):
            n = len(idx)
            raw[:n].copy_(torch.from_numpy(x[idx]))
            mlp._check(lib.hexmlp_pack(int(raw.data_ptr()), n, self.n_in, x.shape[1], int(self.d_x_mean.data_ptr()),
                                       int(self.d_x_inv.data_ptr()), B, net.p_in, int(Xb.data_ptr()),
                                       int(Xt.data_ptr()), st), "pack")
            Tb.zero_()
            Tb[:n, : self.n_out].copy_(torch.from_numpy(yn[idx]))
            return n

        def val_loss():
            total, count = 0.0, 0
            for s in range(0, len(val), B):
                idx = val[s:s + B]
                n = load_batch(idx)
                Y = net.forward(Xb)
                loss = torch.zeros(1, dtype=torch.float32, device="cuda")
                dY = net._workspace(B)["dY"]
                mlp._check(lib.hexmlp_mse_grad(int(Y.data_ptr()), int(Tb.data_ptr()), B, net.p_out, n, self.n_out,
                                               1.0, int(dY.data_ptr()), None, int(loss.data_ptr()), st), "val")
                total += float(loss.item())
                count += n * self.n_out
            return total / max(count, 1)

        rec = NetTraining()
        rec.val_loss_initial = val_loss()
        rec.val_loss_zero = float(np.mean((y[val] / self.y_scale) ** 2))
        t0 = time.perf_counter()
        grads = [t for lay in net.layers for t in (lay.gw, lay.gb)]
        for ep in range(epochs):
            order = rng.permutation(tr)
            ep_loss, ep_n = 0.0, 0
            for b in rank_batches(len(order) // B, rank, world):
                idx = order[b * B:(b + 1) * B]
                n = load_batch(idx)
                loss = net.gradients(Xb, Xt, Tb, n)
                if world > 1:
                    average_gradients(grads, group)
                net.adam(lr * 0.5 * (1.0 + np.cos(np.pi * ep / epochs)))
                rec.steps += 1
                ep_loss += float(loss.item())
                ep_n += n * self.n_out
            rec.train_loss.append(global_mean_loss(ep_loss, ep_n, group if world > 1 else None))
        torch.cuda.synchronize()
        rec.seconds = time.perf_counter() - t0
        net.check()
        rec.val_loss = val_loss()
        return rec


class LearnedStepper:
    """Runs the corrected reduced step on ``reduced``; ``ratio`` full steps
    are the fallback.  ``z_mid`` is the height of every cell level, padded
    layout."""

    def __init__(self, full: HexDycoreDriver, reduced: HexDycoreDriver, col: TrainedNet, edge: TrainedNet, z_mid,
                 *, energy_tol: float = 1e-4, w_growth_tol: float = 0.05, use_network: bool = True,
                 ratio: int = 1):
        import torch

        self.full, self.reduced, self.col, self.edge = full, reduced, col, edge
        self.ratio = int(ratio)
        self.z = z_mid
        self.tol = energy_tol
        self.w_tol = w_growth_tol
        self.use_network = use_network  # False: the same checks and fallback around the bare reduced step
        self.feat = StateFeatures(reduced)
        C_, E_ = self.feat.C, self.feat.E
        self.Cp, self.Ep = mlp.round_up(C_, 128), mlp.round_up(E_, 128)
        self.Xc = torch.empty(self.Cp, col.net.p_in, dtype=torch.bfloat16, device="cuda")
        self.Xe = torch.empty(self.Ep, edge.net.p_in, dtype=torch.bfloat16, device="cuda")
        self.energy = torch.zeros(4, dtype=torch.float64, device="cuda")
        self.fallbacks = 0
        self.flagged = 0
        self.first_fallback = None
        self.steps = 0
        self.last_rel = []
        self.last_growth = []
        self._snap = None
        self._energy_known = False  # slot 0 already holds the energy of the current state

    def reset(self) -> None:
        """Forget counters and the cached energy (after the state was set)."""
        self.fallbacks, self.flagged, self.steps, self.first_fallback = 0, 0, 0, None
        self.last_rel, self.last_growth = [], []
        self._energy_known = False

    def total_energy(self, drv: HexDycoreDriver, slot: int) -> None:
        lib = _lib.load()
        _lib.check(lib.hexdyn_total_energy(drv._handle, _ptr(self.z), C.c_void_p(int(self.energy.data_ptr()) + 16 * slot),
                                           drv._stream_handle()))

    def correct(self) -> None:
        lib, ml = _lib.load(), mlp.load()
        st = mlp._stream()
        f = self.feat
        f.compute(self.reduced)
        for net, raw, X, rows in ((self.col, f.col, self.Xc, f.C), (self.edge, f.edge, self.Xe, f.E)):
            mlp._check(ml.hexmlp_pack(int(raw.data_ptr()), rows, net.n_in, raw.shape[1], int(net.d_x_mean.data_ptr()),
                                      int(net.d_x_inv.data_ptr()), X.shape[0], net.net.p_in, int(X.data_ptr()), None,
                                      st), "pack")
        Yc = self.col.net.forward(self.Xc)
        Ye = self.edge.net.forward(self.Xe)
        _lib.check(lib.hexdyn_apply_increments(self.reduced._handle, _ptr(Yc), Yc.shape[1], _ptr(self.col.d_y_scale),
                                               _ptr(self.col.d_y_shift), _ptr(Ye), Ye.shape[1],
                                               _ptr(self.edge.d_y_scale), _ptr(self.edge.d_y_shift), st))
        _lib.check(lib.hexdyn_rebuild_sidecar(self.reduced._handle, st))

    def step(self) -> bool:
        """One corrected step; returns False when it fell back to the full
        steps (the reduced step's validation flag was set, the energy
        changed by more than the tolerance or the RMS of w grew too fast)."""
        lib = _lib.load()
        snap = self._snap = snapshot_into(self.reduced, self._snap)
        if self._energy_known:
            self.energy[0:2].copy_(self.energy[2:4])  # the last step's result is this step's start
        else:
            self.total_energy(self.reduced, 0)
        self.reduced.step_async(1)
        if self.use_network:
            self.correct()
        self.total_energy(self.reduced, 1)
        flag = C.c_int(0)
        rc = lib.hexdyn_read_flag(self.reduced._handle, self.reduced._stream_handle(), C.byref(flag))
        if rc not in (_lib.HEXDYN_OK, _lib.HEXDYN_E_NUMERIC):
            _lib.check(rc)
        e0, w0, e1, w1 = self.energy.cpu().numpy()
        rel = abs(e1 - e0) / abs(e0)
        growth = np.sqrt(w1 / w0) - 1.0 if w0 > 0 else 0.0
        self.last_rel.append(rel)
        self.last_growth.append(growth)
        self.steps += 1
        ok = bool(flag.value == 0 and np.isfinite(rel) and rel <= self.tol and np.isfinite(growth)
                  and growth <= self.w_tol)
        if flag.value:
            self.flagged += 1
        if not ok and self.first_fallback is None:
            self.first_fallback = self.steps - 1
        self._energy_known = ok
        if not ok:
            self.fallbacks += 1
            restore(self.full, snap)
            self.full.step_async(self.ratio)
            copy_state(self.reduced, self.full)
            rc = lib.hexdyn_read_flag(self.full._handle, self.full._stream_handle(), C.byref(flag))
            if rc == _lib.HEXDYN_E_NUMERIC:
                raise FloatingPointError(f"the full step of the fallback failed at corrected step {self.steps}: "
                                         + _lib.last_error())
            _lib.check(rc)
        return ok
