"""Build the Wang half-resolution known-answer fixture from the reference's test data.

The reference's demo (test_vfs/main.cpp:233-347, the stereoScaling = 2 branch of the
"wang" test) produced ``z16.png`` and ``depth16.png`` (Z and radial depth, uint16 = metres x
256) from ``wang1.png``/``wang2.png`` after ``cv::equalizeHist`` and ``cv::resize`` to
424x400 (main.cpp:306-310), with ``maskHalf.png`` and the ``*WangHalf.flo`` vector fields.
This script repeats that host preprocessing with the Python ``cv2`` bindings and stores
the solver inputs together with the two golden outputs in ``wang_half.npz``.

usage: python make_fixture.py <reference test_vfs directory>
"""
import os
import sys

import cv2
import numpy as np


def read_flo(path):
    b = open(path, "rb").read()
    w, h = np.frombuffer(b, np.int32, 2, 4)
    return np.frombuffer(b, np.float32, int(w) * int(h) * 2, 12).reshape(int(h), int(w), 2).copy()


def main(src, out="wang_half.npz"):
    j = lambda f: os.path.join(src, f)
    im1 = cv2.imread(j("wang1.png"), cv2.IMREAD_GRAYSCALE)
    im2 = cv2.imread(j("wang2.png"), cv2.IMREAD_GRAYSCALE)
    e1 = cv2.resize(cv2.equalizeHist(im1), (424, 400))
    e2 = cv2.resize(cv2.equalizeHist(im2), (424, 400))
    np.savez_compressed(
        out,
        i0=e1, i1=e2,
        mask_u8=cv2.imread(j("maskHalf.png"), cv2.IMREAD_GRAYSCALE),
        tv=read_flo(j("translationVectorWangHalf.flo")),
        cv=read_flo(j("calibrationVectorWangHalf.flo")),
        z16=cv2.imread(j("z16.png"), cv2.IMREAD_UNCHANGED),
        depth16=cv2.imread(j("depth16.png"), cv2.IMREAD_UNCHANGED),
    )
    print("wrote", out)


if __name__ == "__main__":
    main(sys.argv[1], *(sys.argv[2:3]))
