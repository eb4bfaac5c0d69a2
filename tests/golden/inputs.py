"""Readers of the reference test inputs committed beside this file by make_golden.py: the two
fuzz corpora (fuzz_corpus.npz) and the four image fixtures (datasets/*.npy)."""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def corpus(kind: str):
    """(file name, bytes) of every input of the reference's fuzz/corpus/<kind>, in name order."""
    with np.load(os.path.join(HERE, "fuzz_corpus.npz")) as z:
        names = sorted(k for k in z.files if k.startswith(kind + "/"))
        for key in names:
            yield key.split("/", 1)[1], z[key].tobytes()


def datasets():
    """(file name, array) of the reference's datasets/fixtures/*.npy, in name order."""
    folder = os.path.join(HERE, "datasets")
    for name in sorted(os.listdir(folder)):
        if name.endswith(".npy"):
            yield name, np.load(os.path.join(folder, name), allow_pickle=False)
