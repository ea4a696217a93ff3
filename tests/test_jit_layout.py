"""Shared-memory exchanges of the generated pass kernels, checked on the
host from the generated source (no GPU): every exchange's layout is a
bijection onto the tile's 16-byte units, a quarter-warp's accesses fall in
eight distinct bank groups, and where an exchange skips the barrier before
its stores, every thread stores exactly the units it loaded in the previous
exchange (so no thread overwrites data another thread has yet to load)."""
import re

import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from tests.test_plan import mixed_circuit

TERM = re.compile(r"\(\(0u - \(\(\(uint32_t\)(lane|wid) >> (\d)\) & 1u\)\) & 0x([0-9a-f]+)u\)")


def exchanges(kernel, precision):
    """[(barrier_before_store, store_units[thread][k], load_units[thread][k], warp_local)]

    An exchange half declares one pointer per distinct low part m of its
    swizzled offsets, `ptr_m = tile + (pb ^ m)`, and addresses unit
    pb ^ (m | K) as ptr_m[K] (K: the offset's bits above the low three, which
    pb never has); the units below are computed from that form, so the
    checks also cover the pointer arithmetic."""
    decl = r"(?:auto\* const t[sl]\d = (?:tile|pt) \+ \(pb \^ \du\);\n)+"
    if precision == "f64":
        pat = re.compile(r"(__syncthreads\(\);\n)?\{ const uint32_t pb = (0u[^;]*);\n(" + decl +
                         r"(?:ts\d\[\d+u\] = a\[\d+\];\n){16})\}\n"
                         r"(__syncthreads\(\);|__syncwarp\(\);)\n\{ const uint32_t pb = (0u[^;]*);\n(" + decl +
                         r"(?:a\[\d+\] = tl\d\[\d+u\];\n){16})")
    else:
        pat = re.compile(r"(__syncthreads\(\);\n)?\{ ulonglong2\* pt = reinterpret_cast<ulonglong2\*>\(tile\); "
                         r"const uint32_t pb = (0u[^;]*);\n(" + decl + r"(?:ts\d\[\d+u\] = .*\n){8})\}\n"
                         r"(__syncthreads\(\);|__syncwarp\(\);)\n"
                         r"\{ const ulonglong2\* pt = reinterpret_cast<const ulonglong2\*>\(tile\); const uint32_t pb = (0u[^;]*);\n("
                         + decl + r"(?:\{ const ulonglong2 u = tl\d\[\d+u\].*\n){8})")
    out = []
    for m in pat.finditer(kernel):
        def units(expr, body):
            terms = [(w, int(i), int(c, 16)) for w, i, c in TERM.findall(expr)]
            assert len(terms) == 7
            low = {nm: int(v) for nm, v in re.findall(r"auto\* const (t[sl]\d) = \w+ \+ \(pb \^ (\d)u\);", body)}
            accs = re.findall(r"(t[sl]\d)\[(\d+)u\]", body)
            assert len(accs) in (8, 16)
            res = []
            for t in range(128):
                lane, wid = t & 31, t >> 5
                base = 0
                for w, i, c in terms:
                    if ((lane if w == "lane" else wid) >> i) & 1:
                        base ^= c
                res.append([(base ^ low[nm]) + int(k) for nm, k in accs])
            return res
        out.append((m.group(1) is not None, units(m.group(2), m.group(3)), units(m.group(5), m.group(6)),
                    m.group(4) == "__syncwarp();"))
    return out


CASES = [
    ("layered", 20, lambda: C.random_layered(20, 6, 3, initial_h=True), 1),
    ("qft", 20, lambda: C.qft(20), 0),
    ("mixed", 16, lambda: mixed_circuit(16, 200, 8), 0),
    # 26+ qubits: the slot search makes deeper passes with more exchanges
    ("layered26", 26, lambda: C.random_layered(26, 5, 9, initial_h=True), 1),
    ("mixed28", 28, lambda: mixed_circuit(28, 150, 10), 0),
]


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("name,n,make,flags", CASES, ids=[c[0] for c in CASES])
def test_generated_exchanges(name, n, make, flags, precision):
    src, npasses = qb.jit_translate(n, make(), flags=flags, precision=precision)
    kernels = src.split('extern "C"')[1:]
    assert len(kernels) == npasses
    nunits = 2048 if precision == "f64" else 1024
    seen = 0
    for k in kernels:
        xs = exchanges(k, precision)
        # every exchange of the kernel was recognised
        assert len(xs) == (k.count("= a[") // 16 if precision == "f64" else k.count("make_ulonglong2") // 8)
        prev_load = None
        for i, (barrier, st, ld, warp_local) in enumerate(xs):
            if warp_local:
                for w in range(4):
                    warp = range(32 * w, 32 * w + 32)
                    assert sorted(u for t in warp for u in st[t]) == sorted(u for t in warp for u in ld[t]), \
                        "a warp-local exchange loads units another warp stored"
            for side in (st, ld):
                flat = [u for t in side for u in t]
                assert sorted(flat) == list(range(nunits)), "layout is not a bijection"
                for t0 in range(0, 128, 8):   # quarter-warps: 8 distinct bank groups per access
                    for j in range(len(side[0])):
                        assert len({side[t][j] % 8 for t in range(t0, t0 + 8)}) == 8
            if not barrier:
                assert i > 0 and prev_load is not None
                for t in range(128):
                    assert sorted(st[t]) == sorted(prev_load[t]), "store without barrier touches other units"
            prev_load = ld
            seen += 1
    assert seen > 0
