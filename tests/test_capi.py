"""The C-ABI library loads and exports every function include/*.h declares
(no GPU needed: nothing here calls into the device)."""
import ctypes
import glob
import os
import re

import slab

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        txt = re.sub(r"//[^\n]*", "", txt)
        for m in re.finditer(r"\b(slab_[A-Za-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("slab_create", "slab_set_params", "slab_upload_particles", "slab_advance_to_frame", "slab_download_particles",
              "slab_download_grid", "slab_download_max", "slab_conservation", "slab_last_error", "slab_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(slab.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_status_names_without_gpu():
    L = slab.lib()
    assert b"sm_100a" in L.slab_version()
    assert L.slab_status_name(4) == b"SLAB_E_DOMAIN"


def test_null_arguments_are_rejected_without_gpu():
    L = slab.lib()
    assert L.slab_create(None, None, None) == 1
    assert L.slab_set_params(None, None) == 1
    assert L.slab_advance_steps(None, 1, None) == 1
