"""Training and loading of the warm-start network (oflow_net_*).

The network predicts flow at 1/8 resolution (TV-L1 scale 3) from a frame
pair.  It is trained on the GPU by the library's own BF16 forward/backward
kernels (oflow_net_train_step) on synthetic pairs of the 1024x436 generator
(0-3 discs, speeds up to 16 px) labelled by the plain GPU TV-L1 (5 scales x
5 warps x 50 iterations): the label is the plain flow averaged over 8x8 blocks
and divided by 8 (scale-3 pixel units).

  python -m oflow.warmstart --pairs 20000 --epochs 8 --out <file.npz>
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

# (input channels, output channels) per convolution, as in csrc/warmnet.cu
LAYERS = [(16, 32), (32, 32), (32, 64), (64, 64), (64, 96), (96, 96), (96, 128), (224, 96),
          (160, 64), (64, 8)]
# channels that carry signal in layer 0's input (I0, I1, I1-I0; the rest is padding)
_FAN_IN0 = 3
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "warmstart_weights.npz")
W, H = 1024, 436


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights (fan-in 9*C, layer 0 counts its 3 live channels),
    zero biases, last layer scaled by 0.1."""
    rng = np.random.default_rng(seed)
    parts = []
    for i, (cin, cout) in enumerate(LAYERS):
        fan = 9 * (_FAN_IN0 if i == 0 else cin)
        std = np.sqrt(2.0 / fan) * (0.1 if i == len(LAYERS) - 1 else 1.0)
        w = rng.normal(0.0, std, (cout, 3, 3, cin)).astype(np.float32)
        if i == 0:
            w[:, :, :, _FAN_IN0:] = 0.0
        parts += [w.ravel(), np.zeros(cout, np.float32)]
    return np.concatenate(parts)


def save(path: str, params: np.ndarray, meta: dict):
    np.savez_compressed(path, params=params.astype(np.float32), meta=json.dumps(meta))


def load(path: str = WEIGHTS) -> tuple[np.ndarray, dict]:
    d = np.load(path)
    return d["params"].astype(np.float32), json.loads(str(d["meta"]))


def make_dataset(n: int, seed: int, ctx, chunk: int = 32, w: int = W, h: int = H):
    """n labelled pairs on the GPU: frames u8 [n, 2, h, w], targets f32
    [n, oh, ow, 2] (plain TV-L1 flow averaged over 8x8, /8), ground truth
    flow kept for evaluation of the first `chunk` pairs only."""
    import torch
    import torch.nn.functional as F

    import oflow
    from oflow import synth_gpu
    plain = oflow.TVL1Params(nscales=5, max_iterations=50)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)  # order after torch's work
    frames = torch.empty((n, 2, h, w), dtype=torch.uint8, device="cuda")
    oh, ow = -(-h // 8), -(-w // 8)
    targets = torch.empty((n, oh, ow, 2), dtype=torch.float32, device="cuda")
    for s in range(0, n, chunk):
        k = min(chunk, n - s)
        a, b, *_ = synth_gpu.tvl1_pairs(k, w, h, seed=seed + s, ndiscs_max=3, speed_max=16.0)
        frames[s:s + k, 0] = a
        frames[s:s + k, 1] = b
        outs = [(torch.empty((h, w), device="cuda"), torch.empty((h, w), device="cuda"))
                for _ in range(k)]
        oflow.tvl1_batch([(a[i], b[i]) for i in range(k)], plain, ctx, out=outs)
        flow = torch.stack([torch.stack(o) for o in outs])          # [k, 2, h, w]
        tgt = F.avg_pool2d(flow, 8, ceil_mode=True) / 8.0            # [k, 2, oh, ow]
        targets[s:s + k] = tgt.permute(0, 2, 3, 1)
    torch.cuda.synchronize()
    return frames, targets


def train(pairs: int, epochs: int, batch: int, lr: float, seed: int, out: str,
          ckpt_every: int = 500, log=print):
    import torch

    import oflow
    ctx = oflow.Context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    t0 = time.time()
    frames, targets = make_dataset(pairs, seed, ctx)
    log(f"dataset: {pairs} pairs labelled in {time.time() - t0:.1f} s")
    net = oflow.WarmNet(W, H, batch, ctx)
    params = init_params(seed)
    net.set_params(params)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    steps = 0
    hist = []
    t1 = time.time()
    total = epochs * (pairs // batch)
    for ep in range(epochs):
        perm = torch.randperm(pairs, generator=g, device="cuda")
        for i in range(pairs // batch):
            idx = perm[i * batch:(i + 1) * batch]
            f = frames[idx].contiguous()
            t = targets[idx].contiguous()
            # cosine decay of the learning rate
            cur = lr * 0.5 * (1 + np.cos(np.pi * steps / max(total, 1)))
            loss = net.train_step(f, t, float(cur))
            hist.append(loss)
            steps += 1
            if ckpt_every and steps % ckpt_every == 0:
                save(out + ".ckpt.npz", net.get_params(), {"steps": steps})
        log(f"epoch {ep}: mean loss {np.mean(hist[-(pairs // batch):]):.4f} "
            f"({time.time() - t1:.1f} s)")
    p = net.get_params()
    meta = {"pairs": pairs, "epochs": epochs, "batch": batch, "lr": lr, "seed": seed,
            "steps": steps, "final_loss": float(np.mean(hist[-50:])),
            "train_seconds": time.time() - t1,
            "labels": "plain GPU TV-L1, 5 scales x 5 warps x 50, 8x8 average / 8"}
    save(out, p, meta)
    if os.path.exists(out + ".ckpt.npz"):
        os.remove(out + ".ckpt.npz")
    return p, meta


def main(argv=None):
    ap = argparse.ArgumentParser(description="train the TV-L1 warm-start network")
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--out", default=WEIGHTS)
    a = ap.parse_args(argv)
    _, meta = train(a.pairs, a.epochs, a.batch, a.lr, a.seed, a.out,
                    log=lambda *x: print(*x, file=sys.stderr, flush=True))
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
