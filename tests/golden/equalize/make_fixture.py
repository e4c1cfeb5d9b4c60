"""Known answers of cv2.equalizeHist (the routine the reference's SolveStereo calls,
dllhook/vfs.cpp:36-37) for seeded images, including the edge cases: a constant image, a
single pixel, two grey levels, a narrow band and full-range noise.

usage: python make_fixture.py
"""
import cv2
import numpy as np


def main(out="equalize.npz"):
    rng = np.random.default_rng(1234)
    cases = {
        "noise": rng.integers(0, 256, (200, 237), dtype=np.uint8),
        "normal": np.clip(rng.normal(90, 25, (400, 424)), 0, 255).astype(np.uint8),
        "band": rng.integers(120, 131, (61, 77), dtype=np.uint8),
        "two_levels": np.where(rng.random((33, 45)) < 0.3, 10, 200).astype(np.uint8),
        "constant": np.full((17, 19), 77, np.uint8),
        "single": np.array([[201]], np.uint8),
        "t265_like": cv2.GaussianBlur(rng.integers(0, 256, (200, 212), dtype=np.uint8), (7, 7), 2.0),
    }
    d = {}
    for k, v in cases.items():
        d[k + "_in"] = v
        d[k + "_out"] = cv2.equalizeHist(v)
    np.savez_compressed(out, names=np.array(list(cases)), **d)
    print("wrote", out)


if __name__ == "__main__":
    main()
