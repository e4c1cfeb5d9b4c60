"""The host restatement of cv::equalizeHist against cv2's known answers."""
import os

import numpy as np

from oracle.equalize import equalize_hist

FIX = os.path.join(os.path.dirname(__file__), "golden", "equalize", "equalize.npz")


def test_restatement_matches_cv2_known_answers():
    d = np.load(FIX)
    for name in d["names"]:
        assert np.array_equal(equalize_hist(d[f"{name}_in"]), d[f"{name}_out"]), name
