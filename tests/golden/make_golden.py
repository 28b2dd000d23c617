"""Generates the committed golden fixtures under tests/golden/ from the
reference checkout (antequ/fastlinkingnumbers), which exists only in the
development container, never on the GPU hosts:

* ``inputs/<name>.bcc.xz`` — the reference's five regression inputs
  (data/*.bcc verbatim; data/*.obj converted to closed polyline BCC exactly as
  its ``obj2bcc`` does, src/model.cpp:124-264 and :367-452), xz-compressed.
* ``certificates/<name>.txt`` — results/reference_certificates/*.txt.
* ``pairs/<name>.npz`` — per loop pair (i, j), the oracle's FP64 direct-sum
  and Barnes–Hut real-valued sums after PLS + Discretize, and the discretized
  vertex counts, so GPU tests can check real sums without the oracle.
* ``manifest.json`` — expected mean off-integer errors of the default
  Barnes–Hut run (test.sh:4,14,24,34,45) and the oracle's own values.

Usage: python tests/golden/make_golden.py /path/to/reference/checkout
"""
from __future__ import annotations

import json
import lzma
import os
import shutil
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import pyoracle  # noqa: E402

NAMES = ["glove", "knittubeinit", "knittubebroken", "blenderobj", "houdiniobj"]
# test.sh:4,14,24,34,45 — published mean off-integer error of default BH.
PUBLISHED_MEAN_OFF = {"glove": 0.00214443, "knittubeinit": 0.00366683, "knittubebroken": 0.006343,
                      "blenderobj": 0.000668562, "houdiniobj": 0.00138268}


def _is_approx(a, b, prec=1e-12):
    """Eigen's isApprox: |a-b|^2 <= prec^2 * min(|a|^2, |b|^2)."""
    d = [a[k] - b[k] for k in range(3)]
    dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2]
    na = a[0] * a[0] + a[1] * a[1] + a[2] * a[2]
    nb = b[0] * b[0] + b[1] * b[1] + b[2] * b[2]
    return dd <= prec * prec * min(na, nb)


def obj_to_curves(path):
    """Restates Model::ImportFromObjFile (src/model.cpp:124-264): 'v' lines are
    vertices, 'l' lines chain into closed loops; a line whose first vertex is
    not the previous line's last vertex starts a new curve; a repeated closing
    vertex (Houdini) is dropped."""
    ws = " \t\v"
    with open(path) as f:
        lines = f.read().split("\n")
    verts, curves, q = [], [], []
    first_vid = last_vid = -1
    i = 0
    while i < len(lines):
        line = lines[i].strip(ws)
        i += 1
        if not line or line[0] == "#":
            continue
        while line.endswith("\\") and i < len(lines):
            nxt = lines[i].strip(ws)
            i += 1
            line = line[:-1] + " " + nxt
        if len(line) < 2 or line[1] not in ws:
            continue
        toks = [t for t in line[1:].split(" ") if t != ""]
        if line[0] == "v":
            if len(toks) < 3:
                raise ValueError("Obj input: Invalid vertex.")
            verts.append((float(toks[0]), float(toks[1]), float(toks[2])))
        elif line[0] == "l":
            vid = -1
            for t in toks:
                first = vid < 0
                vid = int(t.split("/")[0])
                if first:
                    if vid != last_vid:
                        if len(q) > 1:
                            if last_vid == first_vid or _is_approx(q[-1], q[0]):
                                q.pop()
                            curves.append(q)
                            q = []
                            last_vid = -1
                        q.append(verts[vid - 1])
                        last_vid = vid
                        first_vid = vid
                else:
                    if not (1 <= vid <= len(verts)):
                        raise ValueError("Obj Import: illegal vertex ID.")
                    q.append(verts[vid - 1])
                    last_vid = vid
    if len(q) > 1:
        if last_vid == first_vid or _is_approx(q[-1], q[0]):
            q.pop()
        curves.append(q)
    return curves


def write_bcc_pl(path, curves):
    """BCC writer (src/model.cpp:367-452): 64-byte header, closed loops as
    negative counts, float32 points."""
    total = sum(len(c) for c in curves)
    hdr = b"BCC" + bytes([0x44]) + b"PL" + bytes([3, 1]) + struct.pack("<QQ", len(curves), total)
    hdr += b"\0" * 40
    with open(path, "wb") as f:
        f.write(hdr)
        for c in curves:
            f.write(struct.pack("<i", -len(c)))
            f.write(np.asarray(c, dtype=np.float32).tobytes())


def main(ref):
    os.makedirs(os.path.join(HERE, "inputs"), exist_ok=True)
    os.makedirs(os.path.join(HERE, "certificates"), exist_ok=True)
    os.makedirs(os.path.join(HERE, "pairs"), exist_ok=True)
    manifest = {"published_mean_off_integer_bh": PUBLISHED_MEAN_OFF, "fixtures": {}}
    tmp = os.path.join(HERE, "_tmp")
    os.makedirs(tmp, exist_ok=True)
    for name in NAMES:
        bcc = os.path.join(tmp, name + ".bcc")
        src_bcc = os.path.join(ref, "data", name + ".bcc")
        if os.path.exists(src_bcc):
            shutil.copyfile(src_bcc, bcc)
        else:
            write_bcc_pl(bcc, obj_to_curves(os.path.join(ref, "data", name + ".obj")))
        with open(bcc, "rb") as f, lzma.open(os.path.join(HERE, "inputs", name + ".bcc.xz"), "wb",
                                              preset=9 | lzma.PRESET_EXTREME) as g:
            g.write(f.read())
        shutil.copyfile(os.path.join(ref, "results", "reference_certificates", name + ".txt"),
                        os.path.join(HERE, "certificates", name + ".txt"))
        o = pyoracle.Oracle().load_bcc(bcc)
        text_bh, mean_bh, max_bh = o.certificate(direct=False)
        text_ds, mean_ds, max_ds = o.certificate(direct=True)
        o.prepare(True)
        pairs = o.pairs()
        off, _ = o.polylines()
        small = (len(off) - 1) < 6
        lk_ds, _, _, _ = o.eval_pairs(pyoracle.DIRECT_ONE_ARCTAN if small else pyoracle.DIRECT_FAST,
                                      pairs)
        lk_bh, err_bh, nfar, nleaf = o.eval_pairs(pyoracle.BARNES_HUT, pairs, bh_parallel=small)
        np.savez_compressed(os.path.join(HERE, "pairs", name + ".npz"), pairs=pairs,
                            lk_direct=lk_ds, lk_bh=lk_bh, err_bh=err_bh, far=nfar, leaf=nleaf,
                            vertex_counts=np.diff(off))
        golden = open(os.path.join(HERE, "certificates", name + ".txt")).read()
        manifest["fixtures"][name] = {
            "oracle_bh_matches_golden": text_bh == golden,
            "oracle_directsum_matches_golden": text_ds == golden,
            "oracle_mean_off_integer_bh": mean_bh, "oracle_max_off_integer_bh": max_bh,
            "oracle_mean_off_integer_directsum": mean_ds,
            "curves": int(len(off) - 1), "discretized_vertices": int(off[-1]),
            "pairs": int(len(pairs)), "discretize_rounds": o.rounds,
        }
        print(name, manifest["fixtures"][name])
    shutil.rmtree(tmp)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_golden.py /path/to/reference/checkout")
    main(sys.argv[1])
