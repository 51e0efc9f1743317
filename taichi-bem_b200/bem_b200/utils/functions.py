"""Gauss-Legendre rule on [0,1] (get_gaussion_integration_points_and_weights,
src/BEM_functions/utils/functions.py:5-85): the [-1,1] rule mapped by
p = (x+1)/2, w = w/2, for the orders the reference supports."""
import numpy as np

SUPPORTED = (1, 2, 3, 4, 5, 6, 7, 8, 12)


def get_gaussion_integration_points_and_weights(N: int = 2, np_type=np.float64):
    if N not in SUPPORTED:
        raise NotImplementedError("Please refer N as 2~8 for gaussion interation")
    x, w = np.polynomial.legendre.leggauss(N)
    return [((x + 1.0) / 2.0).astype(np_type), (w / 2.0).astype(np_type)]
