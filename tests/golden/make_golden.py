"""Generates tests/golden/compact_fd6.npz from the reference's own Python
operator, CSS-Python/derivatives.py:32 compact_fd6 (with linalg.py:7
tri_solver), imported from a checkout of the reference.  Run it where the
reference is available; tests only read the committed .npz.

    python tests/golden/make_golden.py <reference checkout>/CSS-Python
    CSS_PYTHON_DIR=<reference checkout>/CSS-Python python tests/golden/make_golden.py

Cases: dtype=0 (whole line; the only mode of compact_fd6 that is correct,
its dtype 1-3 closures do not converge), ibc 0..4, n in {16, 33, 64, 128},
on a sine and on a seeded smooth random field.  For ibc 2/3/4 the Neumann
datum is passed through `darr` as compact_fd6 expects (value per unit of
the whole x-range, i.e. f'(x_end)/dri).
"""
import os
import sys

import numpy as np


class _Darr(np.ndarray):
    # compact_fd6 tests `darr == None`; under numpy 2 that is elementwise, so
    # give the preset array an identity comparison with None.
    def __eq__(self, other):
        if other is None:
            return False
        return np.ndarray.__eq__(self, other)


def main(refdir):
    sys.path.insert(0, refdir)
    import derivatives as d  # the reference module

    rng = np.random.default_rng(20240611)
    cases = []
    for n in (16, 33, 64, 128):
        x1, x2 = 0.75, 1.0
        xs = x1 + (x2 - x1) * np.arange(n) / (n - 1)
        dri = 1.0 / (x2 - x1)
        coef = rng.standard_normal(5)
        fields = {
            "sin": (np.sin(2 * np.pi * (xs - x1) / (x2 - x1)),
                    2 * np.pi / (x2 - x1) * np.cos(2 * np.pi * (xs - x1) / (x2 - x1))),
            "rand": (sum(coef[k] * np.cos((k + 1) * 1.3 * xs + k) for k in range(5)),
                     sum(-coef[k] * (k + 1) * 1.3 * np.sin((k + 1) * 1.3 * xs + k) for k in range(5))),
        }
        for fname, (f, df) in fields.items():
            for ibc in range(5):
                darr = None
                lo = hi = 0.0
                if ibc in (2, 3, 4):
                    darr = np.zeros(n).view(_Darr)
                    if ibc in (2, 4):
                        lo = df[0] / dri
                        darr[0] = lo
                    if ibc in (3, 4):
                        hi = df[-1] / dri
                        darr[n - 1] = hi
                out = d.compact_fd6(dri, f.copy(), 0.0, 0.0, ibc, 0, darr=darr)
                cases.append(dict(n=n, ibc=ibc, field=fname, x=xs, f=f, dri=dri, lo=lo, hi=hi,
                                  out=np.asarray(out, dtype=np.float64)))
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(
        os.path.join(here, "compact_fd6.npz"),
        n=np.array([c["n"] for c in cases]),
        ibc=np.array([c["ibc"] for c in cases]),
        field=np.array([c["field"] for c in cases]),
        dri=np.array([c["dri"] for c in cases]),
        lo=np.array([c["lo"] for c in cases]),
        hi=np.array([c["hi"] for c in cases]),
        f=np.concatenate([c["f"] for c in cases]),
        out=np.concatenate([c["out"] for c in cases]),
    )
    print("wrote %d cases" % len(cases))


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CSS_PYTHON_DIR")
    if not src:
        sys.exit("usage: make_golden.py <reference checkout>/CSS-Python (or set CSS_PYTHON_DIR)")
    main(src)
