"""Layout of the drop-in records and the C ABI surface (no GPU needed)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from sph_b200 import abi, layout, params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sph_isph.h")


def test_record_sizes_match_reference():
    # part1/part2/part3 of class_Cuda_Particle_Array.cuh with Real = float
    assert layout.PART1.itemsize == 152
    assert layout.PART2.itemsize == 52
    assert layout.PART3.itemsize == 164


def test_header_struct_sizes(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include "sph_isph.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(){printf("%zu %zu %zu %zu %zu %zu\\n",sizeof(sph_params),sizeof(sph_part1),'
                   'sizeof(sph_part2),sizeof(sph_part3),sizeof(sph_ppe_stats),offsetof(sph_params,ppe_tol));}')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-I" + os.path.dirname(HEADER), str(src), "-o", str(exe)])
    out = subprocess.check_output([str(exe)]).decode().split()
    assert int(out[0]) == ctypes.sizeof(layout.SphParams)
    assert [int(v) for v in out[1:4]] == [152, 52, 164]
    assert int(out[4]) == ctypes.sizeof(layout.PpeStats)
    assert int(out[5]) == layout.SphParams.ppe_tol.offset


def test_every_params_field_at_the_header_offset(tmp_path):
    # the ctypes mirror and the C struct agree field by field, not only in size
    names = [f for f, _ in layout.SphParams._fields_]
    body = "".join('printf("%%zu\\n", offsetof(sph_params, %s));' % f for f in names)
    src = tmp_path / "off.c"
    src.write_text('#include "sph_isph.h"\n#include <stdio.h>\n#include <stddef.h>\nint main(){' + body + '}')
    exe = tmp_path / "off"
    subprocess.check_call(["gcc", "-I" + os.path.dirname(HEADER), str(src), "-o", str(exe)])
    out = [int(v) for v in subprocess.check_output([str(exe)]).decode().split()]
    assert out == [getattr(layout.SphParams, f).offset for f in names]


def test_prop_tables_fields_at_the_header_offset(tmp_path):
    # sph_prop_tables (the property tables of read_table) and its ctypes mirror
    names = [f for f, _ in layout.PropTables._fields_]
    body = 'printf("%zu\\n", sizeof(sph_prop_tables));' + "".join(
        'printf("%%zu\\n", offsetof(sph_prop_tables, %s));' % f for f in names)
    src = tmp_path / "tab.c"
    src.write_text('#include "sph_isph.h"\n#include <stdio.h>\n#include <stddef.h>\nint main(){' + body + '}')
    exe = tmp_path / "tab"
    subprocess.check_call(["gcc", "-I" + os.path.dirname(HEADER), str(src), "-o", str(exe)])
    out = [int(v) for v in subprocess.check_output([str(exe)]).decode().split()]
    assert out[0] == ctypes.sizeof(layout.PropTables) == 2088
    assert out[1:] == [getattr(layout.PropTables, f).offset for f in names]
    assert layout.TABLE_SIZE == 50 and layout.TABLE_SLOTS == 10


def test_library_loads_and_exports_every_symbol():
    L = abi.lib()
    declared = set()
    import re
    with open(HEADER) as f:
        for line in f:
            m = re.match(r"^(?:const char \*|int64_t |int |void )(sph_\w+)\(", line.strip())
            if m:
                declared.add(m.group(1))
    assert declared == set(abi.SYMBOLS)
    for name in declared:
        assert hasattr(L, name), name


def test_c_defaults_equal_python_defaults():
    c = abi.params_init()
    p = params.default_params()
    for f, _ in layout.SphParams._fields_:
        a, b = getattr(c, f), getattr(p, f)
        if hasattr(a, "__len__"):
            assert list(a) == list(b), f
        else:
            assert a == b, f


def test_domain_setup_c_equals_python():
    from sph_b200 import decks
    P, p = decks.caseh_mini()
    c = abi.params_init()
    c.setf("kappa", p.getf("kappa"))
    abi.domain_setup(c, P)
    for name in ("NI", "NJ", "NK", "num_cells", "num_part2"):
        assert c.geti(name) == p.geti(name), name
    for name in ("x_min", "x_max", "y_min", "y_max", "z_min", "z_max", "dcell", "search_kappa"):
        assert np.float32(c.getf(name)) == np.float32(p.getf(name)), name


def test_create_without_gpu_fails_loudly():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    from sph_b200 import decks
    P, p = decks.caseh_mini(nx=6, ny=4, nz=3)
    with pytest.raises(abi.SphError):
        abi.Simulation(p)


class _FakeDeviceArray:
    """Stands in for a CUDA tensor: only the __cuda_array_interface__ that
    records_arg reads (the pointer is never dereferenced here)."""

    def __init__(self, nbytes, ptr=0x7f0000000000, strides=None, typestr="|u1"):
        self.__cuda_array_interface__ = {"shape": (nbytes // np.dtype(typestr).itemsize,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": strides}


def test_records_arg_passes_device_pointers_through():
    n = 7
    a = _FakeDeviceArray(n * layout.PART1.itemsize)
    ptr, keep, count = abi.records_arg(a, layout.PART1)
    assert ptr.value == 0x7f0000000000 and keep is a and count == n
    assert abi.records_arg(a, layout.PART1, n)[2] == n
    # 4-byte elements, a whole number of records
    b = _FakeDeviceArray(3 * layout.PART2.itemsize, typestr="<f4")
    assert abi.records_arg(b, layout.PART2)[2] == 3


@pytest.mark.parametrize("make,n", [
    (lambda: _FakeDeviceArray(layout.PART1.itemsize * 3 + 4), None),        # not whole records
    (lambda: _FakeDeviceArray(layout.PART1.itemsize * 3), 4),               # wrong count
    (lambda: _FakeDeviceArray(layout.PART1.itemsize * 2, strides=(2,)), None),   # not contiguous
])
def test_records_arg_rejects_malformed_device_arrays(make, n):
    with pytest.raises(ValueError):
        abi.records_arg(make(), layout.PART1, n)


def test_records_arg_host_arrays_keep_their_buffer():
    P = np.zeros(5, layout.PART1)
    ptr, keep, count = abi.records_arg(P, layout.PART1)
    assert count == 5 and keep is P and ptr.value == P.ctypes.data      # no copy of contiguous records
    with pytest.raises(ValueError):
        abi.records_arg(P, layout.PART1, 6)
