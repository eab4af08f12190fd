"""Regenerate the committed golden fixtures from the reference tree.

Run once, in a container that has the reference checkout, naming its
location by argument or by the NEDY_REFERENCE environment variable:

    python tests/golden/make_golden.py <path-to-NEdyson-checkout>

It writes, next to this script:

* calccoeff.json  -- the calculus-weight tables stored by the reference in
  tests/data/calccoeff.h5 (datasets PInterp, PDiff, PInteg, BD, Start, Sigma, w),
  read with the small HDF5 reader below (superblock v0, symbol-table groups,
  contiguous or compact datasets of little-endian float64 -- all this file uses).
* integrals.json  -- the known-answer values of tests/integrals-test.cpp:8-212
  (energy_conv, CTV1, Ctv_tstp, Cles2_tstp, Cles3_tstp), parsed from the test
  source, with the time step each value belongs to and its tolerance.

Nothing at test time reads the reference tree; only these JSON files.
"""
import json
import os
import re
import struct

HERE = os.path.dirname(os.path.abspath(__file__))
REF = None  # the reference checkout, from the command line or NEDY_REFERENCE (see main)


# ---------------------------------------------------------------- HDF5 (tiny)
class H5:
    def __init__(self, path):
        self.d = open(path, "rb").read()
        assert self.d[:8] == b"\x89HDF\r\n\x1a\n", "not an HDF5 file"
        assert self.d[8] == 0, "only superblock version 0 is handled"
        self.so = self.d[13]  # size of offsets
        self.sl = self.d[14]  # size of lengths
        # root symbol table entry follows base/freespace/eof/driver addresses
        p = 24 + 4 * self.so
        self.root = self._entry(p)

    def _u(self, p, n):
        return int.from_bytes(self.d[p:p + n], "little")

    def _entry(self, p):
        name_off = self._u(p, self.so)
        hdr = self._u(p + self.so, self.so)
        ctype = self._u(p + 2 * self.so, 4)
        scratch = p + 2 * self.so + 8
        btree = heap = None
        if ctype == 1:
            btree = self._u(scratch, self.so)
            heap = self._u(scratch + self.so, self.so)
        return dict(name_off=name_off, hdr=hdr, btree=btree, heap=heap)

    def _heap_data(self, heap):
        assert self.d[heap:heap + 4] == b"HEAP"
        return self._u(heap + 8 + 2 * self.sl, self.so)

    def _name(self, heap_data, off):
        e = self.d.index(b"\x00", heap_data + off)
        return self.d[heap_data + off:e].decode()

    def _symbols(self, btree, heap):
        hd = self._heap_data(heap)
        out = {}
        stack = [btree]
        while stack:
            node = stack.pop()
            assert self.d[node:node + 4] == b"TREE"
            level = self.d[node + 5]
            used = self._u(node + 6, 2)
            p = node + 8 + 2 * self.so
            children = []
            for i in range(used):
                p += self.sl  # key
                children.append(self._u(p, self.so))
                p += self.so
            if level > 0:
                stack.extend(children)
                continue
            for snod in children:
                assert self.d[snod:snod + 4] == b"SNOD"
                nsym = self._u(snod + 6, 2)
                q = snod + 8
                for _ in range(nsym):
                    ent = self._entry(q)
                    out[self._name(hd, ent["name_off"])] = ent
                    q += 2 * self.so + 8 + 16
        return out

    def datasets(self):
        return {k: self.read(v["hdr"]) for k, v in self._symbols(self.root["btree"], self.root["heap"]).items()}

    def read(self, hdr):
        assert self.d[hdr] == 1, "object header v1 expected"
        nmsg = self._u(hdr + 2, 2)
        p = hdr + 16
        dims, raw = None, None
        left = nmsg
        while left > 0:
            mtype = self._u(p, 2)
            msize = self._u(p + 2, 2)
            body = p + 8
            if mtype == 0x0001:  # dataspace
                ver = self.d[body]
                rank = self.d[body + 1]
                q = body + (8 if ver == 1 else 4)
                dims = [self._u(q + i * self.sl, self.sl) for i in range(rank)]
            elif mtype == 0x0003:  # datatype: float64 little-endian only
                cls = self.d[body] & 0x0F
                size = self._u(body + 4, 4)
                assert cls == 1 and size == 8, "float64 datasets only"
            elif mtype == 0x0008:  # layout
                ver = self.d[body]
                assert ver == 3
                lclass = self.d[body + 1]
                if lclass == 0:
                    n = self._u(body + 2, 2)
                    raw = self.d[body + 4:body + 4 + n]
                elif lclass == 1:
                    addr = self._u(body + 2, self.so)
                    n = self._u(body + 2 + self.so, self.sl)
                    raw = self.d[addr:addr + n]
                else:
                    raise ValueError("chunked layout not handled")
            elif mtype == 0x0010:  # continuation
                addr = self._u(body, self.so)
                p = addr
                left -= 1
                continue
            p = body + msize
            left -= 1
        n = 1
        for x in dims or [len(raw) // 8]:
            n *= x
        return list(struct.unpack("<%dd" % n, raw[:8 * n]))


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
    h5 = H5(os.path.join(REF, "tests/data/calccoeff.h5"))
    ds = h5.datasets()
    keep = {k: ds[k] for k in ("PInterp", "PDiff", "PInteg", "BD", "Start", "Sigma", "w") if k in ds}
    keep["_source"] = "reference tests/data/calccoeff.h5 (k=5), checked at tests/integration-test.cpp:5-69"
    with open(os.path.join(HERE, "calccoeff.json"), "w") as f:
        json.dump(keep, f, indent=1)
    ints = parse_integrals(os.path.join(REF, "tests/integrals-test.cpp"))
    ints["_source"] = "reference tests/integrals-test.cpp:8-212 with fixtures tests/set_up_g.h:13-242"
    with open(os.path.join(HERE, "integrals.json"), "w") as f:
        json.dump(ints, f, indent=1)
    print({k: len(v) for k, v in keep.items() if isinstance(v, list)},
          {k: len(v) for k, v in ints["cases"].items()})


if __name__ == "__main__":
    main()
