"""Helpers shared by the GPU tests: moving column-major matrices between the
oracle (numpy, Fortran order) and device buffers."""
import numpy as np


def to_dev(A):
    import torch

    A = np.asfortranarray(A)
    return torch.from_numpy(np.ascontiguousarray(A.T)).cuda().reshape(-1)


def from_dev(dA, ld, ncols):
    return np.asfortranarray(dA.view(ncols, ld).T.cpu().numpy())
