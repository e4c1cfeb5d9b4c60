"""Extract the texture-unit golden fixture from the probe programs' output.

The two probes in this folder (``texprobe.cu``, ``texprobe_weights.cu``) were built with
``nvcc -gencode arch=compute_100a,code=sm_100a -O2`` and run on a B200.  They sample
pitch-2D float/float2 textures (normalized coordinates, mirror addressing, linear and point
filtering: the texture setup of every gather in the reference solver) and write
(texture, coordinates, hardware result) records.  This script keeps a compact subset as
``texunit.npz``, which pins the oracle's texture model to the hardware.

usage: python make_fixture.py texprobe.bin texprobe_weights.bin
"""
import struct
import sys

import numpy as np


def load_probe(path):
    b = open(path, "rb").read()
    off = 0
    cases = []
    while off < len(b):
        name = b[off:off + 32].split(b"\0")[0].decode()
        off += 32
        w, h, f2, lin, n = struct.unpack("5i", b[off:off + 20])
        off += 20
        comps = 2 if f2 else 1
        tex = np.frombuffer(b, np.float32, w * h * comps, off).reshape(h, w, comps)
        off += w * h * comps * 4
        xy = np.frombuffer(b, np.float32, n * 2, off).reshape(n, 2)
        off += n * 8
        out = np.frombuffer(b, np.float32, n * comps, off).reshape(n, comps)
        off += n * comps * 4
        cases.append(dict(name=name, w=w, h=h, f2=f2, lin=lin, tex=tex, xy=xy, out=out))
    return cases


def load_weights_probe(path):
    b = open(path, "rb").read()
    n = np.frombuffer(b, np.int32, 1, 0)[0]
    off = 4
    xy = np.frombuffer(b, np.float32, 2 * n, off).reshape(n, 2)
    off += 8 * n
    W, H, S = 53, 50, 64
    recs = []
    for _ in range(7):
        t = np.frombuffer(b, np.float32, S * H, off).reshape(H, S)[:, :W]
        off += 4 * S * H
        o = np.frombuffer(b, np.float32, n, off)
        off += 4 * n
        recs.append((np.ascontiguousarray(t), o))
    return xy, recs


def main(p1, p2, out="texunit.npz"):
    rng = np.random.default_rng(0)
    keep = {}
    k = 0
    for c in load_probe(p1):
        if c["w"] * c["h"] > 250 * 250:
            continue
        n = len(c["xy"])
        sel = np.arange(n) if n <= 6000 else np.sort(rng.choice(n, 6000, replace=False))
        keep[f"c{k}_meta"] = np.array([c["w"], c["h"], c["f2"], c["lin"]], np.int32)
        keep[f"c{k}_tex"] = np.ascontiguousarray(c["tex"])
        keep[f"c{k}_xy"] = np.ascontiguousarray(c["xy"][sel])
        keep[f"c{k}_out"] = np.ascontiguousarray(c["out"][sel])
        k += 1
    xy, recs = load_weights_probe(p2)
    sel = np.concatenate([np.arange(0, 66049, 11), 66049 + np.sort(rng.choice(len(xy) - 66049, 6000, replace=False))])
    for t, o in recs:
        keep[f"c{k}_meta"] = np.array([53, 50, 0, 1], np.int32)
        keep[f"c{k}_tex"] = t[:, :, None]
        keep[f"c{k}_xy"] = np.ascontiguousarray(xy[sel])
        keep[f"c{k}_out"] = np.ascontiguousarray(o[sel][:, None])
        k += 1
    np.savez_compressed(out, ncases=np.int32(k), **keep)
    print("wrote", out, k, "cases")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2], *(sys.argv[3:4]))
