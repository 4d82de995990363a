"""Host restatement of the reference's output-side quantities, for checking the library
(test infrastructure only).

water_table: calc_wtable (Calc_output.f90:20-52) for a grid whose cells are all active --
for each surface column, walk up from the bottom layer (k = nz .. 1), keep the head of each
cell and stop at the first cell whose degree of saturation is not exactly 1; a fully
saturated column ends at its top cell's head.
"""
import numpy as np


def water_table(head, srat, nx, ny, nz):
    h = np.asarray(head, dtype=np.float64).reshape(nz, ny * nx)
    s = np.asarray(srat, dtype=np.float64).reshape(nz, ny * nx)
    out = np.zeros(ny * nx)
    for col in range(ny * nx):
        for k in range(nz - 1, -1, -1):
            out[col] = h[k, col]
            if s[k, col] != 1.0:
                break
    return out
