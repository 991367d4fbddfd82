"""The C-ABI library loads and exports every entry point of include/picomax.h;
without a GPU the device entry points report PMX_ERR_NO_DEVICE (no CPU path)."""
import os
import re

import pytest

from conftest import ROOT, gpu_available

import picomax_b200 as pm
from picomax_b200 import _capi


def header_symbols():
    with open(os.path.join(ROOT, "include", "picomax.h")) as fh:
        text = fh.read()
    return sorted(set(re.findall(r"\b(pmx_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert header_symbols() == sorted(_capi.EXPORTS)


def test_library_exports_every_symbol():
    lib = pm.load()
    for name in header_symbols():
        assert hasattr(lib, name), name


@pytest.mark.skipif(gpu_available(), reason="checks the no-device behaviour")
def test_no_cpu_fallback():
    with pytest.raises(pm.PicomaxError) as e:
        pm.Context(0)
    assert e.value.status == _capi.PMX_ERR_NO_DEVICE


def test_cli_help_and_version():
    import subprocess
    r = subprocess.run([pm.CLI_PATH, "-h"], capture_output=True, text=True)
    assert r.returncode == 0 and "-switch" in r.stdout
    r = subprocess.run([pm.CLI_PATH, "-v"], capture_output=True, text=True)
    assert r.returncode == 0 and "PicoMax version" in r.stdout
