"""C-ABI checks that need no GPU: the library loads, exports every symbol the
public header declares, and the ctypes structures have the header's layout."""
import ctypes as C
import subprocess
import textwrap

import pytest

from spectral_init_b200 import _lib


def test_library_loads_and_exports_every_header_symbol():
    lib = _lib.load()
    declared = _lib.header_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in spectral_init_gpu.h but not exported"
    assert set(_lib._SIGNATURES) == set(declared)
    assert lib.si_abi_version() == 1


def test_config_default_values():
    lib = _lib.load()
    c = _lib.SiConfig()
    lib.si_config_default(C.byref(c))
    assert c.compute_mode == 0 and c.precision == 0 and c.warm_start == 0
    assert c.force_level == -1 and c.rsvd_oversampling == -1


def test_null_context_is_rejected_without_crash():
    lib = _lib.load()
    assert lib.si_ctx_synchronize(None) == _lib.SI_INVALID_ARGUMENT
    assert lib.si_last_error(None) == b"null context"
    out = C.c_void_p()
    # a device index that cannot exist is reported, not aborted
    assert lib.si_ctx_create(1 << 20, C.byref(out)) == _lib.SI_CUDA_ERROR
    assert not out.value


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text(textwrap.dedent("""
        #include <stdio.h>
        #include <stddef.h>
        #include "spectral_init_gpu.h"
        int main(void) {
          printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(si_config), sizeof(si_report), sizeof(si_csr_f32),
                 sizeof(si_csr_f64), sizeof(si_operator), offsetof(si_config, tol), offsetof(si_report, eigenvalues));
          return 0;
        }
    """))
    exe = tmp_path / "sz"
    r = subprocess.run(["gcc", "-I", str(_lib.HEADER_PATH.parent), str(src), "-o", str(exe)], capture_output=True,
                       text=True)
    if r.returncode != 0:
        pytest.skip("gcc unavailable: " + r.stderr)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    want = [C.sizeof(_lib.SiConfig), C.sizeof(_lib.SiReport), C.sizeof(_lib.SiCsrF32), C.sizeof(_lib.SiCsrF64),
            C.sizeof(_lib.SiOperator), _lib.SiConfig.tol.offset, _lib.SiReport.eigenvalues.offset]
    assert got == want
