"""Hand-built SPR structures of dense fronts (test and benchmark helper).

A chain of supernodes j = 1..m with widths S_j where every supernode's row
list is all of its own and later columns, i.e. the factor is dense.  The
arrays follow the layout SPRFC1/SPRFS1/SPRBS1 read (src/SPR/sprfc1.f:165-196,
src/SPR/sprpmp.f:39-48): MTREES = [XSUPER | XSIBL | SIBL | XLINDX | SUPSUP],
MSIFA = [LINDX | XLNZ | XSPLIT].  Supernode j's only child is j-1, so the
extend-add, the outer update (K = S) and the blocked LDL' of a front all run.
"""
import numpy as np


def dense_chain(widths):
    widths = [int(w) for w in widths]
    m = len(widths)
    neq = sum(widths)
    xsuper = np.cumsum([1] + widths)
    xsibl = np.array([1] + [1 + max(0, j) for j in range(m)], dtype=np.int64)
    # supernode j (0-based) has child j-1
    xsibl = np.ones(m + 1, dtype=np.int64)
    sibl = []
    for j in range(m):
        xsibl[j] = len(sibl) + 1
        if j > 0:
            sibl.append(j)          # 1-based child index j-1+1
    xsibl[m] = len(sibl) + 1
    sibl = np.array(sibl + [1] * (m + 1 - len(sibl)), dtype=np.int64)[:m + 1]
    F = [neq - (xsuper[j] - 1) for j in range(m)]
    xlindx = np.cumsum([1] + F)
    lindx = np.concatenate([np.arange(xsuper[j], neq + 1) for j in range(m)]).astype(np.int64)
    sizes = [F[j] * widths[j] - widths[j] * (widths[j] - 1) // 2 for j in range(m)]
    xlnz = np.cumsum([1] + sizes)
    nzerol = int(xlnz[-1] - 1)
    supsup = np.zeros(m, dtype=np.int64)
    mtrees = np.concatenate([xsuper, xsibl, sibl, xlindx, supsup, [1, 0]]).astype(np.int64)
    xsplit = np.ones(m, dtype=np.int64)
    msifa = np.concatenate([lindx, xlnz, xsplit, [0]]).astype(np.int64)
    mspar = np.zeros(60, dtype=np.int64)
    mspar[0] = 4
    mspar[2] = len(msifa)                  # NMSIFA
    mspar[3] = len(mtrees)                 # NTREES
    mspar[7] = neq
    mspar[10] = m                          # NSUPER
    mspar[11] = 0                          # NB
    mspar[12] = max(widths)                # MAXSUP
    mspar[13] = max(F)                     # MFRONT
    mspar[14] = len(lindx)                 # NOFSUB
    mspar[15] = nzerol
    mspar[16] = max(F) * (max(F) + 1) + max(F)        # WSTACK: front + pending update
    mspar[18] = 0                          # NELACT
    mspar[21] = 0                          # NBLOCK
    mspar[44] = 1                          # XSUPER in MTREES
    mspar[45] = 1 + 3 * (m + 1)            # XLINDX in MTREES
    mspar[46] = 1                          # LINDX in MSIFA
    mspar[47] = 1 + len(lindx)             # XLNZ in MSIFA
    return mspar, mtrees, msifa


def pack_dense(A, mspar, mtrees, msifa):
    """SM = [D | LNZ] holding the lower triangle of the dense matrix A."""
    neq = int(mspar[7])
    m = int(mspar[10])
    xsuper = mtrees[:m + 1]
    xlnz = msifa[mspar[47] - 1: mspar[47] + m]
    sm = np.zeros(neq + int(mspar[15]))
    for j in range(m):
        p = xlnz[j] - 1
        for c in range(xsuper[j] - 1, xsuper[j + 1] - 1):
            col = A[c:, c]
            sm[neq + p: neq + p + len(col)] = col
            p += len(col)
    return sm
