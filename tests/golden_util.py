"""Loads the golden fixtures written by tests/golden/make_golden.py."""
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


def load():
    if not os.path.exists(PATH):
        return None
    with np.load(PATH) as z:
        return {k: z[k] for k in z.files}


def codec_cases(fx):
    for k in fx:
        if k.startswith("codec/") and k.endswith("/bytes"):
            _, name, fmt, bw, _ = k.split("/")
            yield name, int(fmt), int(bw)
