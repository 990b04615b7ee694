"""The C-ABI library loads and exports every entry point include/lsmoke_gpu.h declares (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "lsmoke_gpu.h")


def declared_symbols():
    txt = open(HDR).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(lsg_[a-z_0-9]+)\s*\(", txt)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("lsg_reaction_step", "lsg_reaction_step_device", "lsg_mech_load_blob", "lsg_ctx_create"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from laminarsmoke_b200 import lsg
    if not os.path.exists(lsg.LIB_PATH):
        from laminarsmoke_b200.csrc import build
        build.build()
    L = C.CDLL(lsg.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert set(lsg.EXPORTS) <= set(declared_symbols())


def test_options_defaults_and_errors_without_gpu():
    from laminarsmoke_b200 import lsg
    o = lsg.default_options()
    assert (o.rtol, o.atol, o.y_min_T, o.y_max_T, o.max_steps, o.maximum_order) == (1e-7, 1e-12, 200.0, 6000.0, 500000, 5)
    assert (o.alfa2_4, o.alfa2_5, o.energy, o.precision) == (0.8, 0.8, 1, 0)
    L = lsg.lib()
    assert L.lsg_abi_version() == 1
    h = C.c_void_p()
    bad = (C.c_ubyte * 16)(*b"NOTAMECHANISM000")
    assert L.lsg_mech_load_blob(C.cast(bad, C.c_void_p), 16, 0, C.byref(h)) == -2
    assert L.lsg_strerror(-2) == b"mechanism blob could not be read"


def test_property_entry_points_reject_bad_arguments_without_gpu():
    from laminarsmoke_b200 import lsg
    L = lsg.lib()
    has, nt = C.c_int(-1), C.c_int(-1)
    assert L.lsg_mech_transport_info(None, C.byref(has), C.byref(nt), None) == -1
    opt = lsg.PropertyOptions(1, 0, None)
    fields = lsg.PropertyFields()
    y = (C.c_double * 4)()
    assert L.lsg_properties_device(None, 1, 1, C.cast(y, C.c_void_p), C.cast(y, C.c_void_p), 1, None, 101325.,
                                   C.byref(opt), C.byref(fields), 1, None) == -1
    assert L.lsg_properties(None, 1, 1, C.cast(y, C.c_void_p), C.cast(y, C.c_void_p), None, 101325.,
                            C.byref(opt), C.byref(fields)) == -1
    assert [f for f, _ in lsg.PropertyFields._fields_] == list(lsg.PROPERTY_FIELDS)


def test_loader_rejects_inconsistent_transport_arrays_without_gpu():
    """build_transport's size and index checks run before any CUDA call."""
    import numpy as np
    from laminarsmoke_b200 import lsg, mech
    from laminarsmoke_b200.mech import blob
    A, species = blob.unpack(mech.load("h2co")[0])

    def load(arrays):
        data = blob.pack(arrays, species)
        buf = (C.c_ubyte * len(data)).from_buffer_copy(data)
        return lsg.lib().lsg_mech_load_blob(C.cast(buf, C.c_void_p), len(data), 0, C.byref(C.c_void_p()))

    assert load(A) in (0, -3)                                       # consistent: on to the device
    bad = dict(A)
    bad["tr_gamma"] = np.asarray(A["tr_gamma"])[:-4]
    assert load(bad) == -2                                          # LSG_ERR_MECH
    bad = dict(A)
    bad["tr_iteta"] = np.array(list(A["tr_iteta"][:-1]) + [99], np.int32)   # right count, index out of range
    assert load(bad) == -2


def test_loader_rejects_corrupt_headers_and_tables_without_gpu():
    """A huge element count in an array header (which once overflowed the truncation check) and a CSR
    pointer array that decreases are both refused with LSG_ERR_MECH, before any CUDA call."""
    import struct
    import numpy as np
    from laminarsmoke_b200 import lsg, mech
    from laminarsmoke_b200.mech import blob
    data, species = mech.load("h2co")

    def load(d):
        buf = (C.c_ubyte * len(d)).from_buffer_copy(bytes(d))
        return lsg.lib().lsg_mech_load_blob(C.cast(buf, C.c_void_p), len(d), 0, C.byref(C.c_void_p()))

    d = bytearray(data)
    d[16 + 40:16 + 48] = struct.pack("<Q", 1 << 62)          # count of the first array
    assert load(d) == -2
    A, _ = blob.unpack(data)
    bad = dict(A)
    ptr = np.array(A["reac_ptr"])
    ptr[3], ptr[4] = ptr[4], ptr[3]                          # same length and end, decreasing inside
    bad["reac_ptr"] = ptr
    assert load(blob.pack(bad, species)) == -2


_LAYOUT = r"""
#include <stddef.h>
#include <stdio.h>
#include "lsmoke_gpu.h"
#define F(T, m) printf(#T " " #m " %zu\n", offsetof(T, m))
int main(void) {
  printf("lsg_options size %zu\n", sizeof(lsg_options));
  F(lsg_options, rtol); F(lsg_options, max_steps); F(lsg_options, precision); F(lsg_options, alfa2_4);
  F(lsg_options, maximum_order); F(lsg_options, tile); F(lsg_options, autotune); F(lsg_options, jacobian);
  printf("lsg_drg_options size %zu\n", sizeof(lsg_drg_options));
  F(lsg_drg_options, key); F(lsg_drg_options, nkey); F(lsg_drg_options, band_T); F(lsg_drg_options, band_eps);
  F(lsg_drg_options, nbands); F(lsg_drg_options, epsilon0); F(lsg_drg_options, min_T);
  F(lsg_drg_options, first_cell_options_only);
  printf("lsg_property_options size %zu\n", sizeof(lsg_property_options));
  F(lsg_property_options, energy); F(lsg_property_options, simplified_transport); F(lsg_property_options, lewis);
  printf("lsg_property_fields size %zu\n", sizeof(lsg_property_fields));
  F(lsg_property_fields, X); F(lsg_property_fields, cp_species); F(lsg_property_fields, Dsoret);
  return 0;
}
"""


def test_ctypes_structs_match_the_header_layout(tmp_path):
    """The ctypes mirrors of the ABI's structs have the C compiler's sizes and offsets."""
    import shutil
    import subprocess
    from laminarsmoke_b200 import lsg
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    src.write_text(_LAYOUT)
    exe = tmp_path / "layout"
    subprocess.check_call([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    out = subprocess.check_output([str(exe)], text=True).split("\n")
    got = {}
    for line in out:
        parts = line.split()
        if len(parts) == 3:
            got[(parts[0], parts[1])] = int(parts[2])
    classes = {"lsg_options": lsg.Options, "lsg_drg_options": lsg.DrgOptions,
               "lsg_property_options": lsg.PropertyOptions, "lsg_property_fields": lsg.PropertyFields}
    for (struct, field), off in got.items():
        cls = classes[struct]
        if field == "size":
            assert off == C.sizeof(cls), struct
        else:
            assert getattr(cls, field).offset == off, (struct, field)
