"""Trained parameters of the learned PPE preconditioner.

`weights/precond_dambreak.npy` holds the float32 parameter vector (layout of
csrc/learned.cuh) trained by `python -m mps_solvers_b200.train_precond` on
PPE systems of seeded dam-break scenes."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "weights", "precond_dambreak.npy")


def load(path: str = PATH) -> np.ndarray:
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path}: train with `python -m mps_solvers_b200.train_precond`")
    return np.load(path).astype(np.float32)
