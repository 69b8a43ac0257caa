"""The C-ABI library loads on a CPU-only host and exports exactly what include/lbl.h
declares; lbl_config mirrors the reference's config.h defaults.  No GPU calls."""
import ctypes
import math
import os
import re
import subprocess

import pytest

from conftest import ROOT, PKG

import lbl

HEADER = os.path.join(ROOT, "include", "lbl.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?(?:int|void|char\s*\*|const char\*)\s*\**\s*(lbl_\w+)\s*\(", text, re.M)))


def test_header_declares_the_exported_set():
    assert declared_functions() == sorted(lbl.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = lbl.load_library()
    out = subprocess.run(["nm", "-D", "--defined-only", lbl.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (lbl_\w+)$", out, re.M))
    for name in declared_functions():
        assert name in exported, name
        assert hasattr(lib, name)


def test_config_struct_layout_matches_c(tmp_path):
    """sizeof/offsetof of lbl_config from a C compiler equal the ctypes mirror."""
    fields = [f for f, _ in lbl.Config._fields_]
    src = tmp_path / "layout.c"
    body = "".join(f'printf("%zu\\n", offsetof(lbl_config, {f}));' for f in fields)
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "lbl.h"\n'
                   f'int main(void){{printf("%zu\\n", sizeof(lbl_config));{body}return 0;}}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert vals[0] == ctypes.sizeof(lbl.Config)
    for f, off in zip(fields, vals[1:]):
        assert getattr(lbl.Config, f).offset == off, f


def test_config_defaults_follow_reference_config_h():
    c = lbl.config_default("DA_LETKF", 256, 16)
    assert (c.nx, c.ny, c.n_ens) == (256, 256, 16)
    assert c.iiter == 20 and c.iter_main == 40000 and c.spinup == 2000000  # config.h:136-144
    assert c.ioprune == 10 and c.daprune == 10 and c.da_xyprune == 1       # config.h:55-92
    assert c.cs == 0.2 and c.nu == 1e-4 and c.cfl == 0.05                  # lbm.cu:59, config.h:153-157
    assert c.kf == 4 and c.fkf == 5.6 and c.friction_rate == 5e-4          # config.h:161-180
    assert math.isclose(c.h_ref, 2 * math.pi) and c.u_ref == 1 and c.rho_ref == 1
    assert c.force_seed == 1991 and c.obs_seed == 334                      # data.cu:294, io.cu:321
    assert c.jacobi_max_sweeps == 100 and c.jacobi_tol == 1e-6             # eigensolver_wrapper.hpp:192-193
    assert c.letkf_covinf == 1.0 and c.compat_stale_v == 1
    assert c.abi_version == lbl.ABI_VERSION


def test_config_overrides_and_unknown_key():
    c = lbl.config_default("OBSERVE", 128, 1, da_xyprune=4, obs_error_u=0.2)
    assert c.da_xyprune == 4 and c.obs_error_u == 0.2 and c.iiter == 10
    with pytest.raises(KeyError):
        lbl.config_default("NATURE", 256, 1, not_a_field=1)


def test_version_string():
    assert "sm_100a" in lbl.version()


def test_oracle_config_mirror_matches_the_product():
    """The oracle's own lbl_config mirror and config.h defaults (used by the CPU
    reference arm, which must not load liblbl) equal the product's field for field."""
    import oracle
    assert [f for f, _ in oracle.Config._fields_] == [f for f, _ in lbl.Config._fields_]
    assert ctypes.sizeof(oracle.Config) == ctypes.sizeof(lbl.Config)
    for f, _ in lbl.Config._fields_:
        assert getattr(oracle.Config, f).offset == getattr(lbl.Config, f).offset, f
    for mode, nx, m in (("NATURE", 256, 1), ("OBSERVE", 128, 1), ("DA_LETKF", 512, 64), ("DA_NUDGING", 64, 4)):
        a = oracle.config_default(mode, nx, m, cs=0.1, tau=0.51).as_dict()
        b = lbl.config_default(mode, nx, m, cs=0.1, tau=0.51).as_dict()
        assert a == b, (mode, nx, m)
