"""Committed golden fixtures (tests/golden/*.npz) made by make_golden.py from the
reference renderer compiled as the oracle."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def path(name: str) -> str:
    return os.path.join(HERE, f"{name}.npz")


def load(name: str) -> dict:
    with np.load(path(name), allow_pickle=False) as z:
        return {k: z[k] for k in z.files}
