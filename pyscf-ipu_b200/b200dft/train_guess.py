"""Train the learned initial-guess network on converged densities that the engine generates.

    python -m b200dft.train_guess --nmol 50000 --epochs 12 --out <weights.npz>

Data: seeded molecules of the batched distribution (1-9 heavy atoms C/N/O/F, H to valence) with
seeds disjoint from the benchmark's; each chunk is converged by ``RKSEngine.run_converged``
(mixed precision, MINAO start) and its density matrices become the targets.  Training: Adam,
mini-batches of molecules, cosine learning-rate decay, all on the GPU through csrc/learned.cu.
"""
import argparse
import os
import time
import numpy as np
import torch

from .mole import Mole
from .molgen import config3_batch
from .engine import RKSEngine
from .learned import GuessNet, Batch

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "guess_net.npz")


def generate(nmol, seed, chunk=4096, level=0, log=print):
    """(atom strings, converged D per molecule (host float64 arrays)) for nmol molecules"""
    atoms = config3_batch(nmol, seed=seed)
    Ds = []
    for c0 in range(0, nmol, chunk):
        mols = [Mole(s) for s in atoms[c0:c0 + chunk]]
        t0 = time.time()
        eng = RKSEngine(mols, level=level, precision="mixed")
        res = eng.run_converged(max_its=40)
        D = eng.D.cpu().numpy()
        for mi in range(len(mols)):
            Ds.append(eng.plan.unpack(D, mi).copy())
        conv = res["converged"].cpu().numpy()
        log(f"  generated {c0 + len(mols)}/{nmol} ({conv.mean():.3f} converged, {time.time() - t0:.1f}s)")
        eng.close()
        del eng
        torch.cuda.empty_cache()
    return atoms, Ds


def make_batches(atoms, Ds, bs, device="cuda"):
    out = []
    for b0 in range(0, len(atoms), bs):
        mols = [Mole(s) for s in atoms[b0:b0 + bs]]
        B = Batch(mols, device=device)
        Dt = np.zeros(B.n_mat)
        for mi, D in enumerate(Ds[b0:b0 + bs]):
            o = int(B.mat_off[mi])
            Dt[o:o + D.size] = D.reshape(-1)
        out.append((B, torch.from_numpy(Dt).to(device)))
    return out


def train(net, batches, epochs, lr=1e-3, lr_min=1e-5, log=print, val=None):
    steps = epochs * len(batches)
    k = 0
    for ep in range(epochs):
        perm = np.random.default_rng(ep).permutation(len(batches))
        tot = 0.0
        for bi in perm:
            B, Dt = batches[bi]
            cur = lr_min + 0.5 * (lr - lr_min) * (1 + np.cos(np.pi * k / max(1, steps)))
            tot += net.train_step(B, Dt, lr=cur).item()
            k += 1
        msg = f"  epoch {ep + 1}/{epochs}: train mse {tot / len(batches):.3e}"
        if val:
            msg += f"  val mse {evaluate(net, val):.3e}"
        log(msg)
    return net


def evaluate(net, batches):
    tot = 0.0
    for B, Dt in batches:
        z, y, _ = net.forward(B)
        D = torch.zeros(B.n_mat, dtype=torch.float64, device=net.device)
        loss, _, _ = net.assemble(B, z, y, D, Dt)
        tot += loss.item()
    return tot / max(1, len(batches))


def save(net, path=WEIGHTS):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, params=net.params.cpu().numpy(), n_params=net.n_params, hl=net.hl, hr=net.hr)


def load(path=WEIGHTS, device="cuda"):
    d = np.load(path)
    # files written before the hidden widths were recorded hold the 256 / 512 network
    hl = int(d["hl"]) if "hl" in d else 256
    hr = int(d["hr"]) if "hr" in d else 512
    net = GuessNet(device=device, hl=hl, hr=hr)
    if int(d["n_params"]) != net.n_params:
        raise ValueError("weights do not match the network layout")
    net.params.copy_(torch.from_numpy(d["params"]).to(net.device))
    return net


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nmol", type=int, default=50000)
    ap.add_argument("--val", type=int, default=1024)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--bs", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=7001)
    ap.add_argument("--out", default=WEIGHTS)
    a = ap.parse_args(argv)
    t0 = time.time()
    atoms, Ds = generate(a.nmol + a.val, a.seed)
    print(f"data: {len(atoms)} molecules in {time.time() - t0:.1f}s")
    tr = make_batches(atoms[:a.nmol], Ds[:a.nmol], a.bs)
    va = make_batches(atoms[a.nmol:], Ds[a.nmol:], a.bs)
    print(f"batches built at {time.time() - t0:.1f}s")
    net = GuessNet(seed=0)
    train(net, tr, a.epochs, lr=a.lr, val=va)
    save(net, a.out)
    print(f"saved {a.out} ({net.n_params} parameters) at {time.time() - t0:.1f}s")


if __name__ == "__main__":
    main()
