"""Trains the graph network of the learned preconditioner on the GPU and
writes its weights next to this file (weights/gnn_near_spai.f32 plus a JSON
record of the run).

Data: seeded synthetic sphere meshes (N from 1350 to 8262 basis functions)
with random jitter (up to 0.1 of the cell), radius (0.8-1.25), frequency
(0.5-3) and material (isotropic, anisotropic tensor or Gaussian-profile
permittivity).  Each visit assembles the VIE
matrix, solves one plane-wave right-hand side by LU for the solution term of
the objective, and takes a few Adam steps with fresh random probes.

    python buff-em_b200/train_gnn.py [--meshes 200] [--epochs 3] [--out PATH]
"""
import argparse
import json
import math
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import buffem  # noqa: E402
import meshgen  # noqa: E402

DEFAULT_OUT = os.path.join(HERE, "weights", "gnn_near_spai.f32")


def random_material(rng):
    u = rng.random()
    if u < 0.45:
        return buffem.Material(eps=complex(rng.uniform(2, 12), rng.uniform(0, 1.5))), "iso"
    if u < 0.8:
        d = rng.uniform(2, 10, size=3)
        off = rng.uniform(-0.8, 0.8)
        t = np.diag(d).astype(complex) + 1j * rng.uniform(0, 1) * np.eye(3)
        t[0, 1] = t[1, 0] = off
        return buffem.Material(kind=buffem.BG_MAT_CONST_TENSOR, tensor=t), "tensor"
    return buffem.Material(kind=buffem.BG_MAT_GAUSSIAN, eps=complex(rng.uniform(2, 6), rng.uniform(0, 0.5)),
                           amp=complex(rng.uniform(1, 5), 0), width=rng.uniform(0.3, 1.0)), "gaussian"


def make_dataset(n_meshes, seed, meshdir):
    rng = np.random.default_rng(seed)
    items = []
    for s in range(n_meshes):
        n = int(rng.integers(5, 10))
        items.append(dict(n=n, jitter=float(rng.uniform(0, 0.1)), radius=float(rng.uniform(0.8, 1.25)),
                          omega=float(rng.uniform(0.5, 3.0)), seed=seed * 100000 + s,
                          mat_seed=int(rng.integers(1 << 31))))
    return items


def visit(item, meshdir):
    path = meshgen.cached_sphere(meshdir, item["n"], item["radius"], item["jitter"], item["seed"])
    mat, _ = random_material(np.random.default_rng(item["mat_seed"]))
    G = buffem.SWGGeometry(meshfiles=path, materials=mat)
    w = item["omega"]
    A = G.AssembleVIEMatrix(w)
    b = G.AssembleRHSVector(w, buffem.PlaneWave([1, 0, 0], [0, 0, 1]))
    L = G.AssembleVIEMatrix(w)
    L.LUFactorize()
    x = b.copy()
    L.LUSolve(x)
    del L
    return G, A, b, x


def evaluate(net, meshdir, sizes=(10, 12), omega=1.0):
    out = []
    for n in sizes:
        G = buffem.SWGGeometry(meshfiles=meshgen.cached_sphere(meshdir, n, 1.0, 0.1, 4242 + n),
                               materials=buffem.Material(eps=6 + 0.5j))
        A = G.AssembleVIEMatrix(omega)
        B = np.zeros((G.TotalBFs, 2), complex, order="F")
        B[:, 0] = G.AssembleRHSVector(omega, buffem.PlaneWave([1, 0, 0], [0, 0, 1]))
        B[:, 1] = G.AssembleRHSVector(omega, buffem.PlaneWave([0, 1, 0], [1, 0, 0]))
        _, sj = buffem.GMRESSolve(A, B, buffem.Preconditioner.jacobi(A), tol=1e-10, restart=50, maxit=3000)
        _, sl = buffem.GMRESSolve(A, B, buffem.Preconditioner.learned(G, A, omega, net), tol=1e-10, restart=50,
                                  maxit=3000)
        out.append({"N": G.TotalBFs, "steps_jacobi": int(sj[0]), "steps_learned": int(sl[0])})
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--meshes", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--steps-per-visit", type=int, default=3)
    ap.add_argument("--probes", type=int, default=8)
    ap.add_argument("--probe-power", type=int, default=8,
                    help="every other step maps the probes this many times through z <- z - A D^-1 z")
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--lam", type=float, default=0.5)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--meshdir", default=os.path.join(tempfile.gettempdir(), "buffem_gnn_meshes"))
    args = ap.parse_args(argv)
    items = make_dataset(args.meshes, args.seed, args.meshdir)
    rng = np.random.default_rng(args.seed + 1)
    net = buffem.GNN(seed=args.seed)
    total = args.epochs * len(items) * args.steps_per_visit
    step = 0
    t0 = time.time()
    curve = []
    for ep in range(args.epochs):
        order = rng.permutation(len(items))
        ep_loss = []
        for k in order:
            G, A, b, x = visit(items[k], args.meshdir)
            N = G.TotalBFs
            for _ in range(args.steps_per_visit):
                lr = 1e-4 + 0.5 * (args.lr - 1e-4) * (1 + math.cos(math.pi * step / total))
                Z = rng.normal(size=(N, args.probes)) + 1j * rng.normal(size=(N, args.probes))
                power = args.probe_power if step % 2 else 0
                ep_loss.append(net.train_step(G, A, items[k]["omega"], Z, b, x, lam=args.lam, lr=lr,
                                              probe_power=power))
                step += 1
            del A, G
        curve.append(float(np.mean(ep_loss)))
        print(f"epoch {ep}: mean objective {curve[-1]:.4f}  ({time.time() - t0:.0f} s)", flush=True)
    params = net.params()
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    params.astype("<f4").tofile(args.out)
    ev = evaluate(net, args.meshdir)
    record = {"params": int(params.size), "seed": args.seed, "meshes": args.meshes, "epochs": args.epochs,
              "steps": step, "probes": args.probes, "probe_power": args.probe_power, "lambda": args.lam,
              "lr_peak": args.lr,
              "epoch_objective": curve, "train_seconds": time.time() - t0, "held_out": ev}
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(record, f, indent=1)
    print(json.dumps(record), flush=True)


if __name__ == "__main__":
    main()
