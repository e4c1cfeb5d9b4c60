"""Histogram equalisation restated on the host (TEST INFRASTRUCTURE ONLY).

The reference's C-ABI SolveStereo equalises both input images with cv::equalizeHist before
solving (dllhook/vfs.cpp:36-37).  That routine lives in OpenCV (4.5.1, the version the
reference names in readme.md:10), imgproc/src/histogram.cpp, not in the reference itself; its
published algorithm is restated here:
  hist = 256-bin histogram, i = first non-empty bin;
  if hist[i] == total: every pixel becomes i;
  else scale = 255 / (total - hist[i]) (float), lut[i] = 0 and for j > i
       lut[j] = round-half-even(float(cumsum(hist[i+1..j])) * scale), saturated to 0..255.
Pinned against cv2.equalizeHist outputs in tests/golden/equalize.
"""
import numpy as np


def equalize_hist(img: np.ndarray) -> np.ndarray:
    img = np.ascontiguousarray(img, np.uint8)
    hist = np.bincount(img.ravel(), minlength=256).astype(np.int64)
    total = img.size
    if total == 0:
        return img.copy()
    i = int(np.argmax(hist > 0))
    if hist[i] == total:
        return np.full_like(img, i)
    scale = np.float32(255.0) / np.float32(total - hist[i])
    lut = np.zeros(256, np.uint8)
    s = 0
    for j in range(i + 1, 256):
        s += int(hist[j])
        v = np.float32(s) * scale
        lut[j] = np.uint8(min(max(int(np.rint(v)), 0), 255))
    return lut[img]
