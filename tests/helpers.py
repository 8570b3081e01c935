"""Shared helpers of the parity tests."""
import numpy as np


def system_blocks(sys, vertex_of_row=None):
    """{(row vertex, col vertex): 9 floats} and b by vertex, from an exported system."""
    rowptr, cols, vals = sys["rowptr"], sys["cols"], sys["vals"].reshape(-1, 9)
    n = rowptr.size - 1
    vor = np.arange(n) if vertex_of_row is None else vertex_of_row
    blocks = {}
    for r in range(n):
        i = int(vor[r])
        for k in range(int(rowptr[r]), int(rowptr[r + 1])):
            blocks[(i, int(vor[int(cols[k])]))] = vals[k]
    b = np.zeros((n, 3), np.float32)
    b[vor] = sys["b"].reshape(-1, 3)
    return blocks, b


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))
