"""Full-size certificate fixtures of the benchmark workloads, from the FP64
direct sum of every potentially linked pair (run on a B200).

The reference's certificate is the direct sum, rounded
(linking_number_certificate.cpp:241-338, :294-322). The FP64 GPU direct sum
(`fln_linking_numbers`, method directsum, FLN_PREC_FP64) restates
ComputeLinkingNumberDirectFast in FP64 and is held within 1e-9 of the CPU
oracle by tests/test_gpu_parity.py; over the full workloads it takes minutes
(polymer ~7, held_out_20M ~11, mixed_batch ~25 on one B200), where the CPU
oracle would take hours. So this script writes, per workload:

  configs/<name>.txt   the certificate (the reference's text format)
  configs/<name>.npz   the FP64 real sum of every pair (in the prepared pair
                       order), the digest of the prepared polylines and
                       pairs, sizes, seed and device time

Two steps, so that a long workload can run over several GPU calls:

  # on the GPU: FP64 direct sum of parts [a, b) of K work-balanced parts
  python tests/golden/make_config_certs.py run --config polymer --parts 8 \
      --range 0:8 --out /tmp/fixtures
  # anywhere: check and merge the parts into tests/golden/configs/
  python tests/golden/make_config_certs.py merge --config polymer --src /tmp/fixtures

The workloads are seeded (workloads.named); the digest pins the prepared
polylines and pairs, so the test that reads these fixtures first checks that
it regenerated the same input.
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from fastlinkingnumbers_b200 import workloads  # noqa: E402

OUT_DIR = os.path.join(HERE, "configs")
SEEDS = {"polymer": 3, "held_out_20M": 3, "mixed_batch": 3}


def prepare(name: str, engine):
    from fastlinkingnumbers_b200 import Model
    off, xyz, desc = workloads.named(name, SEEDS[name])
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    del xyz
    poff, pxyz, pairs, rounds = m.Prepare(True, engine=engine)
    return poff, pxyz, pairs, rounds, desc


def split(work: np.ndarray, parts: int):
    """Contiguous ranges of pairs with about equal direct-sum work."""
    c = np.concatenate([[0.0], np.cumsum(work)])
    cuts = np.searchsorted(c, np.linspace(0, c[-1], parts + 1), side="left")
    cuts[0], cuts[-1] = 0, len(work)
    return [(int(cuts[k]), int(cuts[k + 1])) for k in range(parts)]


def run(args):
    from fastlinkingnumbers_b200 import Engine
    from fastlinkingnumbers_b200 import _native as N
    os.makedirs(args.out, exist_ok=True)
    eng = Engine(0)
    t0 = time.time()
    poff, pxyz, pairs, rounds, desc = prepare(args.config, eng)
    dig = workloads.digest(poff, pxyz, pairs)
    n = np.diff(poff).astype(np.float64)
    work = n[pairs[:, 0]] * n[pairs[:, 1]]
    print(f"{args.config}: {len(pairs)} pairs, {poff[-1]} segments, {work.sum():.4g} segment pairs, "
          f"digest {dig}, prepared in {time.time() - t0:.1f} s", flush=True)
    if args.save_pairs:
        np.save(os.path.join(args.out, f"{args.config}.pairs.npy"), pairs)
    a, b = (int(x) for x in args.range.split(":"))
    for k, (lo, hi) in enumerate(split(work, args.parts)):
        if not (a <= k < b):
            continue
        t1 = time.time()
        lk, _, _ = eng.linking_numbers(pxyz, poff, pairs[lo:hi], "directsum", precision=N.PREC_FP64,
                                       fp64_margin=0.0)
        s = eng.stats()
        path = os.path.join(args.out, f"{args.config}.part{k:03d}of{args.parts:03d}.npz")
        np.savez(path, lo=lo, hi=hi, lk=lk, digest=dig, kernel_ms=s["ms_main_kernel"],
                 segment_pairs=work[lo:hi].sum())
        print(f"  part {k}: pairs [{lo}, {hi}), {work[lo:hi].sum():.3g} segment pairs, kernel "
              f"{s['ms_main_kernel'] / 1e3:.1f} s, wall {time.time() - t1:.1f} s", flush=True)
    meta = {"config": args.config, "seed": SEEDS[args.config], "description": desc, "digest": dig,
            "pairs": int(len(pairs)), "segments": int(poff[-1]), "loops": int(len(poff) - 1),
            "discretize_rounds": int(rounds), "segment_pairs": float(work.sum()), "parts": args.parts}
    with open(os.path.join(args.out, f"{args.config}.meta.json"), "w") as f:
        json.dump(meta, f, indent=1)
    eng.close()


def merge(args):
    with open(os.path.join(args.src, f"{args.config}.meta.json")) as f:
        meta = json.load(f)
    parts = sorted(glob.glob(os.path.join(args.src, f"{args.config}.part*of{meta['parts']:03d}.npz")))
    if len(parts) != meta["parts"]:
        raise SystemExit(f"{len(parts)} of {meta['parts']} parts present")
    lk = np.full(meta["pairs"], np.nan)
    ms = 0.0
    for p in parts:
        z = np.load(p)
        if str(z["digest"]) != meta["digest"]:
            raise SystemExit(f"{p}: digest differs")
        lk[int(z["lo"]):int(z["hi"])] = z["lk"]
        ms += float(z["kernel_ms"])
    if not np.all(np.isfinite(lk)):
        raise SystemExit("missing or non-finite pairs")
    # The pairs themselves are regenerated by Prepare and pinned by the digest;
    # the certificate needs them, so they come from the last part's run.
    pairs = None
    pz = os.path.join(args.src, f"{args.config}.pairs.npy")
    if os.path.exists(pz):
        pairs = np.load(pz)
    if pairs is None:
        raise SystemExit(f"{pz} missing (written by `run --save-pairs`)")
    text = workloads.certificate_text(meta["loops"], pairs, lk)
    os.makedirs(OUT_DIR, exist_ok=True)
    with open(os.path.join(OUT_DIR, f"{args.config}.txt"), "w") as f:
        f.write(text)
    off_int = np.abs(lk - np.sign(lk) * np.floor(np.abs(lk) + 0.5))
    meta.update({"fp64_kernel_s": round(ms / 1e3, 1), "nonzero_links": text.count("\n") - 1,
                 "min_margin": float(0.5 - off_int.max()), "mean_off_integer": float(off_int.mean())})
    np.savez_compressed(os.path.join(OUT_DIR, f"{args.config}.npz"), lk=lk, meta=json.dumps(meta))
    print(json.dumps(meta, indent=1))


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    r = sub.add_parser("run")
    r.add_argument("--config", required=True, choices=sorted(SEEDS))
    r.add_argument("--parts", type=int, default=8)
    r.add_argument("--range", default="0:1000000")
    r.add_argument("--out", required=True)
    r.add_argument("--save-pairs", type=int, default=1)
    m = sub.add_parser("merge")
    m.add_argument("--config", required=True, choices=sorted(SEEDS))
    m.add_argument("--src", required=True)
    args = ap.parse_args()
    if args.cmd == "run":
        run(args)
    else:
        merge(args)


if __name__ == "__main__":
    main()
