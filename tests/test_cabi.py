"""The C ABI library loads and exports every symbol include/b200chem.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared():
    txt = (ROOT / "include" / "b200chem.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(b200chem_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared()
    for n in ("b200chem_create", "b200chem_set_typvals", "b200chem_react", "b200chem_react_flat",
              "b200chem_destroy", "b200chem_eval_rhs", "b200chem_eval_jac", "b200chem_inst_rr",
              "b200chem_t_from_hy"):
        assert n in names


def test_library_exports_all_declared_symbols():
    from pelelmex_b200 import build
    lib = ctypes.CDLL(str(build.build()))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.b200chem_version() == 3


def test_struct_layouts_match_header():
    from pelelmex_b200 import _lib
    assert ctypes.sizeof(_lib.Array4) == 8 + 3 * 8 + 6 * 4
    assert ctypes.sizeof(_lib.BoxView) == 24 + 7 * ctypes.sizeof(_lib.Array4)
    assert ctypes.sizeof(_lib.Opts) == 2 * 8 + 12 * 4  # two doubles and twelve int32 fields
    assert ctypes.sizeof(_lib.ChemBox) == 24 + 11 * ctypes.sizeof(_lib.Array4) + 8
    assert ctypes.sizeof(_lib.ForceBox) == 24 + 7 * ctypes.sizeof(_lib.Array4)


def test_null_arguments_of_the_box_list_calls_are_rejected_without_gpu():
    from pelelmex_b200 import _lib
    L = _lib.load()
    assert L.b200chem_react_force(None, None, 0, 1e-6, None) == -1
    assert L.b200chem_advance_chemistry(None, None, 0, 1e-6, None, None, None) == -1


def test_null_handle_is_rejected_without_gpu():
    from pelelmex_b200 import _lib
    L = _lib.load()
    dt = ctypes.c_double(1e-6)
    assert L.b200chem_react(None, None, 0, ctypes.byref(dt), None, None, None, None) == -1
    assert b"bad arguments" in L.b200chem_last_error()


def test_mechanism_digest_selects_generated_code():
    """The library's FNV-1a digest of a mechanism description equals the
    generator's, so the generated right-hand side of each bundled mechanism
    is the one react uses; any change to the description selects none."""
    import numpy as np
    from pelelmex_b200 import _lib, mechanism as M, mechgen
    L = _lib.load()
    for name in ("synth_h2_9", "synth_ch4_21", "synth_c12_53"):
        flat = M.flatten(M.builtin(name))
        desc = flat.ctypes_desc()
        d = L.b200chem_mechanism_digest(ctypes.byref(desc))
        assert d == mechgen.mechanism_digest(flat)
        assert L.b200chem_generated_species(d) == flat.n_species
        flat.arrays["arr"][0, 0] = np.nextafter(flat.arrays["arr"][0, 0], 0.0)  # one ulp off one rate
        desc2 = flat.ctypes_desc()
        d2 = L.b200chem_mechanism_digest(ctypes.byref(desc2))
        assert d2 != d and d2 == mechgen.mechanism_digest(flat)
        assert L.b200chem_generated_species(d2) == 0
