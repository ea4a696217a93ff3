"""Host side of the generated pass kernels (no GPU): the generator emits one
kernel per tile pass, its text depends on the pass structure only (not on
angle values), and every emitted kernel compiles with NVRTC for sm_100a."""
import re

import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from tests.test_plan import mixed_circuit


def kernels(src):
    return re.findall(r'extern "C" __global__ void __launch_bounds__\(128, \d+\) (qoa_jit_pass_[0-9a-f]{16})', src)


@pytest.mark.parametrize("n,make,flags", [
    (13, lambda: C.random_layered(13, 5, 1, initial_h=True), 1),
    (14, lambda: C.qft(14), 0),
    (13, lambda: mixed_circuit(13, 120, 2), 0),
])
def test_one_kernel_per_pass_and_it_compiles(n, make, flags):
    ops = make()
    src, npasses = qb.jit_translate(n, ops, flags=flags, compile=True)
    names = kernels(src)
    assert npasses > 0
    assert len(names) == npasses
    # passes of the plan (QINIT-free op lists: the same scheduler)
    assert qb.plan(n, ops, flags=flags)["npasses"] >= npasses


@pytest.mark.parametrize("n,make,flags", [
    (13, lambda: C.random_layered(13, 5, 3, initial_h=True), 1),
    (13, lambda: mixed_circuit(13, 120, 4), 0),
])
def test_complex64_kernels_compile(n, make, flags):
    src, npasses = qb.jit_translate(n, make(), flags=flags, compile=True, precision="f32")
    assert npasses > 0
    assert len(re.findall(r"qoa_jit_pass32_[0-9a-f]{16}\(float2\*", src)) == npasses


def test_text_depends_on_structure_not_angles():
    n = 13
    def circ(a):
        return [C.Op(C.H, [q]) for q in range(n)] + [C.Op(C.RZ, [q], a * (q + 1)) for q in range(n)] + \
               [C.Op(C.CPHASE, [q, (q + 4) % n], a) for q in range(n)]
    s1, _ = qb.jit_translate(n, circ(0.37))
    s2, _ = qb.jit_translate(n, circ(1.21))
    assert s1 == s2
    s3, _ = qb.jit_translate(n, circ(0.37)[:-1])
    assert s3 != s1


def test_literal_exchange_and_condition_forms():
    # CNOTs with lane-bit controls and targets outside the first registers
    # give thread conditions and exchanges; both appear as literals
    n = 14
    ops = [C.Op(C.H, [q]) for q in range(n)] + [C.Op(C.CNOT, [q, (q + 7) % n]) for q in range(n)]
    src, npasses = qb.jit_translate(n, ops, compile=False)
    assert npasses >= 1
    assert re.search(r"auto\* const ts\d = tile \+ \(pb \^ \du\);", src)  # exchange pointers: literal offsets
    assert re.search(r"ts\d\[\d+u\] = a\[\d+\];", src)
    assert re.search(r"\(\(tw & 0x[0-9a-f]+u\) == 0x[0-9a-f]+u\)", src)


def test_bad_sizes_fail_cleanly():
    with pytest.raises(qb.QoaError):
        qb.jit_translate(8, C.qft(8))
    with pytest.raises(qb.QoaError):
        qb.jit_translate(40, C.qft(4))


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_batch_form_compiles(precision):
    """The batch (arena) form: one kernel per pass over a job list, the
    rotation form read at run time; it compiles and its text does not
    depend on rotation angles."""
    n = 13
    def circ(a):
        return [C.Op(C.H, [q]) for q in range(n)] + [C.Op(C.RY, [q], a * (q + 1)) for q in range(n)] + \
               [C.Op(C.CZ, [q, (q + 1) % n]) for q in range(n)] + [C.Op(C.RX, [q], 2.9 - a * q) for q in range(n)]
    src1, np1 = qb.jit_translate(n, circ(0.21), compile=True, precision=precision, arena=True)
    src2, np2 = qb.jit_translate(n, circ(1.37), precision=precision, arena=True)
    assert np1 == np2 and np1 > 0
    assert src1 == src2
    assert "const qoa::ArenaJob J = jobs[blockIdx.x >> 2];" in src1
