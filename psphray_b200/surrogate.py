"""The chemistry surrogate of the non-isothermal ticks: training data logged
by the integrator, a network trained on the GPU by libpsg's own forward and
backward kernels (psg_mlp_grad, psg_mlp_adam), and its installation into
the ticks (psg_set_surrogate), where it runs in BF16 on the tensor cores and
falls back per particle to the integrator.

No counterpart in the reference, which integrates every particle's step
with LSODA (src/solve.c:170-224).

    python -m psphray_b200.surrogate --out psphray_b200/data/surrogate_lognormal128.npz

trains on the log-normal workload's first ticks and writes the network.
torch serves as device memory and for shuffling rows; the network's
arithmetic is libpsg's.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import api

NFEAT = 5                     # inputs used of the 8 in a row
NPARAM = 4866
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_PATH = os.path.join(HERE, "data", "surrogate_lognormal128.npz")


def init_params(seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0, np.sqrt(2.0 / NFEAT), (64, 8))
    W1[:, NFEAT:] = 0.0
    parts = [W1, np.zeros(64), rng.normal(0, np.sqrt(2.0 / 64), (64, 64)), np.zeros(64),
             rng.normal(0, np.sqrt(1.0 / 64), (2, 64)), np.zeros(2)]
    p = np.concatenate([a.ravel() for a in parts]).astype(np.float32)
    assert len(p) == NPARAM
    return p


class Surrogate:
    """A trained network with its input and output normalisation."""

    def __init__(self, params, x_mu, x_sd, y_mu, y_sd, meta=None):
        self.params = np.ascontiguousarray(params, np.float32)
        self.x_mu = np.ascontiguousarray(x_mu, np.float32)
        self.x_sd = np.ascontiguousarray(x_sd, np.float32)
        self.y_mu = np.ascontiguousarray(y_mu, np.float32)
        self.y_sd = np.ascontiguousarray(y_sd, np.float32)
        self.meta = meta or {}

    def save(self, path: str):
        np.savez(path, params=self.params, x_mu=self.x_mu, x_sd=self.x_sd, y_mu=self.y_mu, y_sd=self.y_sd,
                 meta=json.dumps(self.meta))

    @classmethod
    def load(cls, path: str = DEFAULT_PATH) -> "Surrogate":
        with np.load(path) as z:
            return cls(z["params"], z["x_mu"], z["x_sd"], z["y_mu"], z["y_sd"], json.loads(str(z["meta"])))

    def install(self, ctx: api.Context, tol: float = 1e-3):
        ptr = lambda a: a.ctypes.data
        ctx._check(api.lib().psg_set_surrogate(ctx.h, ptr(self.params), ptr(self.x_mu), ptr(self.x_sd),
                                                ptr(self.y_mu), ptr(self.y_sd), C.c_float(tol)),
                   "psg_set_surrogate")

    @staticmethod
    def uninstall(ctx: api.Context):
        ctx._check(api.lib().psg_set_surrogate(ctx.h, None, None, None, None, None, C.c_float(0)),
                   "psg_set_surrogate")

    def predict(self, ctx: api.Context, rows):
        """The installed network (tensor cores) on raw input rows (torch
        [n, 8] float32 on the device); returns [n, 2] outputs."""
        import torch
        y = torch.empty((rows.shape[0], 2), dtype=torch.float32, device=rows.device)
        ctx._check(api.lib().psg_surrogate_forward(ctx.h, C.c_void_p(rows.data_ptr()), rows.shape[0],
                                                   C.c_void_p(y.data_ptr())), "psg_surrogate_forward")
        return y


def collect(ctx: api.Context, rays_fn, nray: int, nticks_per_call: int, calls: int, first_tick: int,
            tick_time: float, cap: int):
    """Runs `calls` batches of ticks with the update log on; returns the
    logged rows (torch [n, 8], device) and the next tick."""
    import torch
    rows = torch.zeros((cap, 8), dtype=torch.float32, device=f"cuda:{ctx.device}")
    count = torch.zeros(1, dtype=torch.int64, device=rows.device)
    ctx._check(api.lib().psg_set_update_log(ctx.h, C.c_void_p(rows.data_ptr()), cap, C.c_void_p(count.data_ptr())),
               "psg_set_update_log")
    tick = first_tick
    try:
        for _ in range(calls):
            ctx.run_ticks(rays_fn(tick, nticks_per_call), nray, nticks_per_call, tick, tick_time)
            tick += nticks_per_call
    finally:
        ctx._check(api.lib().psg_set_update_log(ctx.h, None, 0, None), "psg_set_update_log")
    n = min(int(count.item()), cap)
    return rows[:n], tick


def fit(ctx: api.Context, rows, epochs: int = 8, batch: int = 8192, lr: float = 2e-3, seed: int = 1,
        val_frac: float = 0.02, log=print) -> tuple[Surrogate, list]:
    """Trains on logged rows with libpsg's gradient and Adam kernels."""
    import torch
    dev = rows.device
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    # the extreme 0.5% of each target (a particle ionised or heated through
    # in one step) are left to the integrator: the residual check rejects
    # them anyway, and they would dominate the squared error
    y_all = rows[:, NFEAT:NFEAT + 2].double()
    q = torch.quantile(y_all[torch.randperm(rows.shape[0], generator=g, device=dev)[:1_000_000]],
                       torch.tensor([0.005, 0.995], dtype=torch.float64, device=dev), dim=0)
    keep = ((y_all >= q[0]) & (y_all <= q[1])).all(1)
    rows = rows[keep]
    feat = rows[:, :NFEAT].double()
    y = rows[:, NFEAT:NFEAT + 2].double()
    x_mu, x_sd = feat.mean(0), feat.std(0).clamp_min(1e-6)
    y_mu, y_sd = y.mean(0), y.std(0).clamp_min(1e-9)
    X = torch.zeros((rows.shape[0], 8), dtype=torch.float32, device=dev)
    X[:, :NFEAT] = ((feat - x_mu) / x_sd).float()
    T = ((y - y_mu) / y_sd).float().contiguous()
    perm = torch.randperm(rows.shape[0], generator=g, device=dev)
    nval = max(1, int(val_frac * rows.shape[0]))
    Xv, Tv = X[perm[:nval]].contiguous(), T[perm[:nval]].contiguous()
    Xt, Tt = X[perm[nval:]].contiguous(), T[perm[nval:]].contiguous()
    ntr = Xt.shape[0]
    params = torch.from_numpy(init_params(seed)).to(dev)
    m = torch.zeros_like(params)
    v = torch.zeros_like(params)
    grad = torch.zeros(NPARAM + 1, dtype=torch.float32, device=dev)
    L = api.lib()
    P = lambda t: C.c_void_p(t.data_ptr())
    steps_per_epoch = ntr // batch
    total = epochs * steps_per_epoch
    hist = []
    step = 0
    t0 = time.time()
    for ep in range(epochs):
        order = torch.randperm(ntr, generator=g, device=dev)
        for i in range(steps_per_epoch):
            idx = order[i * batch:(i + 1) * batch]
            xb, tb = Xt[idx].contiguous(), Tt[idx].contiguous()
            ctx._check(L.psg_mlp_grad(ctx.h, P(params), P(xb), P(tb), batch, P(grad), None), "psg_mlp_grad")
            step += 1
            rate = lr * (0.03 + 0.97 * 0.5 * (1 + np.cos(np.pi * step / total)))
            ctx._check(L.psg_mlp_adam(ctx.h, P(params), P(grad), P(m), P(v), C.c_float(rate), C.c_float(0.9),
                                      C.c_float(0.999), C.c_float(1e-8), step), "psg_mlp_adam")
        ctx._check(L.psg_mlp_grad(ctx.h, P(params), P(Xv), P(Tv), Xv.shape[0], P(grad), None), "psg_mlp_grad")
        val = float(grad[NPARAM].item()) / Xv.shape[0]
        hist.append(val)
        log(f"epoch {ep}: validation mse {val:.3e} (normalised), {time.time() - t0:.1f} s")
    s = Surrogate(params.cpu().numpy(), x_mu.float().cpu().numpy(), x_sd.float().cpu().numpy(),
                  y_mu.float().cpu().numpy(), y_sd.float().cpu().numpy(),
                  meta={"rows": int(rows.shape[0]), "epochs": epochs, "batch": batch, "lr": lr,
                        "val_mse": hist[-1] if hist else None})
    return s, hist


FLOP_PER_ROW = 2 * (16 * 64 + 64 * 64 + 64 * 16)     # the three tensor-core layers as padded


def forward_bench(n: int, reps: int = 20):
    """Times the shipped network on the tensor cores (psg_surrogate_forward)
    over n rows of inputs drawn around the training distribution."""
    import torch
    s = Surrogate.load()
    from .units import Units
    ctx = api.Context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)     # events and kernels on one stream
    ctx.set_physics(api.Physics(Units(hmf=1.0), isothermal=False))
    s.install(ctx)
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    rows = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
    rows[:, :NFEAT] = torch.from_numpy(s.x_mu).cuda() + torch.from_numpy(s.x_sd).cuda() * torch.randn(
        (n, NFEAT), generator=g, device="cuda")
    y = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    run = lambda: ctx._check(api.lib().psg_surrogate_forward(ctx.h, C.c_void_p(rows.data_ptr()), n,
                                                             C.c_void_p(y.data_ptr())), "psg_surrogate_forward")
    for _ in range(3):
        run()
    torch.cuda.synchronize()
    ms = 0.0
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        e1.synchronize()
        ms += e0.elapsed_time(e1) / reps
    print(json.dumps({"rows": n, "ms": ms, "rows_per_s": n / ms * 1e3,
                      "tflops": n * FLOP_PER_ROW / ms / 1e9, "flop_per_row": FLOP_PER_ROW}))
    ctx.close()


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=DEFAULT_PATH)
    ap.add_argument("--forward-bench", type=int, default=0, help="time the shipped network on N rows and exit")
    ap.add_argument("--calls", type=int, default=4, help="batches of 8 ticks logged")
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--cap", type=int, default=60_000_000)
    args = ap.parse_args()
    if args.forward_bench:
        forward_bench(args.forward_bench)
        return
    from . import fields
    w = fields.make_workload("lognormal128")
    phys = api.Physics(w.field.units, isothermal=False)
    ctx = api.Context(0)
    ctx.set_physics(phys)
    ctx.load(w.field)
    ctx.build_tree(8)
    rows, _ = collect(ctx, w.schedule.rays_for_ticks, w.schedule.nray, 8, args.calls, 1, w.tick_time, args.cap)
    print(f"logged {rows.shape[0]} particle updates")
    s, _ = fit(ctx, rows, epochs=args.epochs)
    s.save(args.out)
    print(f"wrote {args.out}")
    ctx.close()


if __name__ == "__main__":
    main()
