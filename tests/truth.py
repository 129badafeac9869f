"""Long-double evaluations of the assembly routines, as a reference for the
rounding error of the FP64 results.

Each routine's independent numpy transcription (tests/test_*_assembly.py) is
fed the same double inputs converted to long double (x87, 64-bit mantissa),
so its formulas and their order are evaluated with ~1e-19 relative rounding,
the transcendental functions through numpy's long double ufuncs; the
tridiagonal solve runs in long double too.  Comparing the oracle (the FP64
restatement of the reference) and the GPU against this shows how far each is
from the exact result of the same formulas."""
import numpy as np

from test_comp_assembly import comp_numpy
from test_minor_assembly import minor_numpy
from test_oplus_assembly import oplus_numpy
from test_settei_assembly import settei_numpy

LD = np.longdouble


def ld(F):
    """The fields of a routine as long double arrays (constants stay double)."""
    return {k: (np.asarray(v, dtype=LD) if isinstance(v, np.ndarray) and v.dtype == np.float64 else v)
            for k, v in F.items()}


def thomas(a, b, c, f, k2):
    """Rows 1..k2 of the tridiagonal solve, trsolv_ng's recurrence, in the
    inputs' precision; rows past k2 are zero."""
    nk = a.shape[0]
    x = np.zeros_like(f)
    w1 = np.empty_like(f)
    w2 = np.empty_like(f)
    w3 = np.empty_like(f)
    w1[0] = b[0]
    w3[0] = f[0] / w1[0]
    for k in range(1, k2):
        w2[k - 1] = c[k - 1] / w1[k - 1]
        w1[k] = b[k] - a[k] * w2[k - 1]
        w3[k] = (f[k] - a[k] * w3[k - 1]) / w1[k]
    x[k2 - 1] = w3[k2 - 1]
    for k in range(k2 - 2, -1, -1):
        x[k] = w3[k] - w2[k] * x[k + 1]
    assert nk >= k2
    return x


def comp_truth(F, C):
    upd = comp_numpy(ld(F), C)[0]
    return [upd[i] for i in range(3)]


def minor_truth(F, C):
    p, q, r, f = minor_numpy(ld(F), C)
    return thomas(p, q, r, f, p.shape[0])


def oplus_truth(F, C):
    p, q, r, ex, x2p, x2d, fe, fn = oplus_numpy(ld(F), C)
    nk = p.shape[0]
    x = thomas(p, q, r, ex, nk - 1)
    x[nk - 1] = x[nk - 2] * x[nk - 2] / x[nk - 3]
    return [x, x2p, x2d, fe, fn]


def settei_truth(F, C, qtotal):
    Fl = ld(F)
    p, q, r, rhs, q2, lei, lin = settei_numpy(Fl, C, np.asarray(qtotal, dtype=LD))
    nk = p.shape[0]
    x = thomas(p, q, r, rhs, nk - 1)
    x[:nk - 1] = np.power(x[:nk - 1], LD(2. / 7.))   # the double exponent the code writes
    x[nk - 1] = x[nk - 2] * x[nk - 2] / x[nk - 3]
    tn = Fl["tn"]
    te = np.maximum(x, tn)
    ti = np.maximum((Fl["qji_ti"] * Fl["xnmbar"] / C["avo"] + lei * te + lin * tn) / (lei + lin), tn)
    return [te, ti, q2]


def rel(got, truth):
    """max over columns of |got - truth| / max|truth| (the column's norm)."""
    t = np.asarray(truth, dtype=LD)
    scale = np.maximum(np.max(np.abs(t), axis=0), LD(1e-300))
    return float(np.max(np.abs(np.asarray(got, dtype=LD) - t) / scale))
