"""Regenerate the committed golden fixtures from the reference tree.

Run once, in a container that has the reference checkout, naming its
location by argument or by the NEDY_REFERENCE environment variable:

    python tests/golden/make_golden.py <path-to-NEdyson-checkout>

It writes, next to this script:

* calccoeff.json  -- the calculus-weight tables stored by the reference in
  tests/data/calccoeff.h5 (datasets PInterp, PDiff, PInteg, BD, Start, Sigma, w),
  read with the package's HDF5 reader (nedyson_b200/h5io.py).
* gfree_const.json -- the free propagator G0_from_h0 of the reference's free-test
  (tests/data/Gfree_const.h5, tests/free-test.cpp:8-42): the first k+1 time steps of
  GR, GL, GTV and the Matsubara component.
* integrals.json  -- the known-answer values of tests/integrals-test.cpp:8-212
  (energy_conv, CTV1, Ctv_tstp, Cles2_tstp, Cles3_tstp), parsed from the test
  source, with the time step each value belongs to and its tolerance.

Nothing at test time reads the reference tree; only these JSON files.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = None  # the reference checkout, from the command line or NEDY_REFERENCE (see main)


# ---------------------------------------------------------------- HDF5
# the package's reader (superblock v0, symbol-table groups, contiguous / compact data)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from nedyson_b200.h5io import H5File  # noqa: E402


# ----------------------------------------------------------- integrals goldens
def parse_integrals(path):
    src = open(path).read()
    cases = {}
    for m in re.finditer(r'TEST_CASE\("([^"]+)"\)\{(.*?)\n\}', src, re.S):
        name, body = m.group(1), m.group(2)
        if name.startswith("TTI"):
            continue
        vals = []
        if name == "Energy Integral":
            for t, v, tol in re.findall(
                    r"energy_conv\((\d+), S, G, beta, dt\);\s*REQUIRE\(std::abs\(res \+ ([0-9.eE+-]+)\) < ([0-9.eE+-]+)\)", body):
                vals.append(dict(t=int(t), value=[-float(v), 0.0], tol=float(tol)))
        elif name == "CTV1":
            for t, re_, im_, tol in re.findall(
                    r"CTV1\(res.data\(\), S, Scc, G, (\d+), dt\);\s*REQUIRE\(std::abs\(res.sum\(\) - cplx\(([^,]+),([^)]+)\)\) < ([0-9.eE+-]+)\)", body):
                vals.append(dict(t=int(t), value=[float(re_), float(im_)], tol=float(tol)))
        elif name == "Ctv_tstp":
            for t, re_, im_, tol in re.findall(
                    r"Ctv_tstp\((\d+), G, G, Gcc, S, Scc, beta, dt\);\s*REQUIRE\(std::abs\(ZRowVectorMap\(G.tvptr\(\d+,0\), \(Ntau\+1\) \* Nao \* Nao\).sum\(\) - cplx\(([^,]+),([^)]+)\)\) < ([0-9.eE+-]+)\)", body):
                vals.append(dict(t=int(t), value=[float(re_), float(im_)], tol=float(tol)))
        elif name in ("Cles2_tstp", "Cles3_tstp"):
            pat = (r"Cles2_tstp\(G, Gcc, S, Scc, (\d+), dt, res.data\(\)\);" if name == "Cles2_tstp"
                   else r"Cles3_tstp\(S, Scc, G, Gcc, (\d+), beta, res.data\(\)\);")
            for t, nsum, re_, im_, tol in re.findall(
                    pat + r"\s*REQUIRE\(std::abs\(ZRowVectorMap\(res.data\(\), \((\d+)\+1\) \* Nao \* Nao\).sum\(\) - cplx\(([^,]+),([^)]+)\)\) < ([0-9.eE+-]+)\)", body):
                vals.append(dict(t=int(t), nsum=int(nsum) + 1, value=[float(re_), float(im_)], tol=float(tol)))
        cases[name] = vals
    return dict(Nt=50, Ntau=30, Nao=2, beta=1.5, dt=0.02, k=5, sig=-1, cases=cases)


def main():
    global REF
    import sys
    REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NEDY_REFERENCE")
    if not REF:
        sys.exit("usage: make_golden.py <path-to-NEdyson-checkout>  (or set NEDY_REFERENCE)")
    h5 = H5File(os.path.join(REF, "tests/data/calccoeff.h5"))
    keep = {k: [float(v) for v in h5["/" + k]] for k in ("PInterp", "PDiff", "PInteg", "BD", "Start", "Sigma", "w")
            if "/" + k in h5}
    keep["_source"] = "reference tests/data/calccoeff.h5 (k=5), checked at tests/integration-test.cpp:5-69"
    with open(os.path.join(HERE, "calccoeff.json"), "w") as f:
        json.dump(keep, f, indent=1)
    ints = parse_integrals(os.path.join(REF, "tests/integrals-test.cpp"))
    ints["_source"] = "reference tests/integrals-test.cpp:8-212 with fixtures tests/set_up_g.h:13-242"
    with open(os.path.join(HERE, "integrals.json"), "w") as f:
        json.dump(ints, f, indent=1)
    # free propagator of a constant h0 (reference tests/free-test.cpp:8-42): G0_from_h0 with
    # Nt=20, Ntau=30, nao=2, beta=9, dt=0.1, mu=1, h0 = [[1, -3], [-3, 2]]; the test compares
    # the first k+1 = 6 time steps and the Matsubara component
    fr = H5File(os.path.join(REF, "tests/data/Gfree_const.h5"))
    nao, ntau = 2, 30
    es, nk = nao * nao, 6
    tri = nk * (nk + 1) // 2
    cut = {"GR": tri * es, "GL": tri * es, "GTV": nk * (ntau + 1) * es, "GM": (ntau + 1) * es}
    gfree = {"_source": "reference tests/data/Gfree_const.h5, checked at tests/free-test.cpp:8-42",
             "Nt": 20, "Ntau": ntau, "nao": nao, "beta": 9.0, "dt": 0.1, "mu": 1.0, "h0": [[1.0, -3.0], [-3.0, 2.0]],
             "k": 5, "tol_norm": 1e-10}
    for k, n in cut.items():
        v = fr["/" + k][:n]
        gfree[k] = [[float(z.real), float(z.imag)] for z in v]
    with open(os.path.join(HERE, "gfree_const.json"), "w") as f:
        json.dump(gfree, f, indent=0)
    print({k: len(v) for k, v in keep.items() if isinstance(v, list)},
          {k: len(v) for k, v in ints["cases"].items()})


if __name__ == "__main__":
    main()
