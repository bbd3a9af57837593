"""ctypes binding of libqb (include/qb.h).

The shared library is built in-tree by ``q_b200/build.py`` (or
``__graft_entry__.build()``) into ``q_b200/libqb.so``.  There is no fallback:
if the library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(_HERE)
LIB_PATH = os.environ.get("QB_LIBRARY", os.path.join(_HERE, "libqb.so"))
INCLUDE = os.path.join(REPO, "include")

QB_NE = 29
QB_NEQ = 15
QB_MAX_STATES = 10

STATUS = {
    0: "QB_OK", 1: "QB_ERR_ARG", 2: "QB_ERR_IO", 3: "QB_ERR_PARSE", 4: "QB_ERR_UNSUPPORTED",
    5: "QB_ERR_SHAKE", 6: "QB_ERR_NAN", 7: "QB_ERR_LIST_OVERFLOW", 8: "QB_ERR_TIMEOUT",
    9: "QB_ERR_CUDA", 10: "QB_ERR_STATE",
}

# Energy vector names in qb_energy_index order (nrgy.f90:43-49).
E_NAMES = [
    "potential", "kinetic", "LRF",
    "p_bond", "p_angle", "p_torsion", "p_improper",
    "w_bond", "w_angle", "w_torsion", "w_improper",
    "q_bond", "q_angle", "q_torsion", "q_improper",
    "pp_el", "pp_vdw", "pw_el", "pw_vdw", "ww_el", "ww_vdw", "qx_el", "qx_vdw",
    "rst_total", "rst_fix", "rst_shell", "rst_protein", "rst_solvent_radial", "rst_water_pol",
]
EQ_NAMES = [
    "lambda", "total", "bond", "angle", "torsion", "improper",
    "qx_el", "qx_vdw", "qq_el", "qq_vdw", "qp_el", "qp_vdw", "qw_el", "qw_vdw", "restraint",
]


class QBError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def _struct_from_header(path: str, name: str) -> type:
    """Build a ctypes.Structure for `typedef struct <name> {...} <name>;` by
    reading the declaration in the public header, so the layout has a single
    source of truth."""
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    defines = {k: int(v) for k, v in re.findall(r"#define\s+(\w+)\s+(\d+)\b", src)}
    m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), src, flags=re.S)
    if not m:
        raise RuntimeError(f"{name} not found in {path}")
    base = {"int": C.c_int, "double": C.c_double, "float": C.c_float,
            "unsigned char": C.c_ubyte, "signed char": C.c_byte, "unsigned int": C.c_uint}
    fields = []
    for decl in m.group(1).split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        const = decl.startswith("const ")
        if const:
            decl = decl[6:]
        tname = None
        for t in sorted(base, key=len, reverse=True):
            if decl.startswith(t + " ") or decl.startswith(t + "*"):
                tname = t
                break
        if tname is None:
            raise RuntimeError(f"unparsed field: {decl}")
        rest = decl[len(tname):]
        for item in rest.split(","):
            item = item.strip()
            ptr = item.startswith("*")
            item = item.lstrip("*").strip()
            arr = re.match(r"(\w+)\[(\w+)\]", item)
            if arr:
                dim = arr.group(2)
                fields.append((arr.group(1), base[tname] * (int(dim) if dim.isdigit() else defines[dim])))
            elif ptr:
                fields.append((item, C.POINTER(base[tname])))
            else:
                fields.append((item, base[tname]))
    return type(name, (C.Structure,), {"_fields_": fields})


SysView = _struct_from_header(os.path.join(INCLUDE, "qb_system.h"), "qb_sysview")


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("device", C.c_int), ("verbose", C.c_int),
                ("reserved", C.c_int * 5)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libqb not built: {LIB_PATH} is missing (run `python -m q_b200.build`)")
    lib = C.CDLL(LIB_PATH)
    vp, ip, dp, fp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_float)
    sig = {
        "qb_version": (C.c_int, [C.c_char_p, C.c_size_t]),
        "qb_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
        "qb_device_count": (C.c_int, [ip]),
        "qb_open": (C.c_int, [C.c_char_p, C.POINTER(Options), C.POINTER(vp)]),
        "qb_open_override": (C.c_int, [C.c_char_p, C.POINTER(Options), dp, C.c_int, C.c_int,
                                       C.POINTER(vp)]),
        "qb_get_view": (C.c_int, [vp, C.POINTER(SysView)]),
        "qb_close": (None, [vp]),
        "qb_batch_create": (C.c_int, [C.POINTER(vp), C.c_int, C.POINTER(Options), C.POINTER(vp)]),
        "qb_batch_run": (C.c_int, [vp, C.c_int]),
        "qb_batch_final_energy": (C.c_int, [vp]),
        "qb_batch_evaluate": (C.c_int, [vp, C.c_int]),
        "qb_batch_get_coords_all": (C.c_int, [vp, dp]),
        "qb_batch_set_coords_all": (C.c_int, [vp, dp]),
        "qb_batch_get_velocities_all": (C.c_int, [vp, dp]),
        "qb_batch_set_velocities_all": (C.c_int, [vp, dp]),
        "qb_batch_history_all": (C.c_int, [vp, C.c_int, C.c_int, C.POINTER(C.c_int), dp, C.POINTER(C.c_size_t)]),
        "qb_batch_step_count": (C.c_int, [vp, C.POINTER(C.c_longlong)]),
        "qb_batch_box": (C.c_int, [vp, C.c_int, dp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
        "qb_batch_run_timed": (C.c_int, [vp, C.c_int, dp, C.POINTER(C.c_longlong)]),
        "qb_peak_flops": (C.c_int, [C.c_int, C.c_int, dp]),
        "qb_batch_energies": (C.c_int, [vp, C.c_int, dp, dp]),
        "qb_batch_temperature": (C.c_int, [vp, C.c_int, dp]),
        "qb_batch_gradient": (C.c_int, [vp, C.c_int, dp]),
        "qb_batch_get_coords": (C.c_int, [vp, C.c_int, dp]),
        "qb_batch_set_coords": (C.c_int, [vp, C.c_int, dp]),
        "qb_batch_get_velocities": (C.c_int, [vp, C.c_int, dp]),
        "qb_batch_set_velocities": (C.c_int, [vp, C.c_int, dp]),
        "qb_batch_get_theta_corr": (C.c_int, [vp, C.c_int, fp, C.c_int]),
        "qb_batch_history": (C.c_int, [vp, C.c_int, C.c_int, ip, ip, dp, dp]),
        "qb_batch_offdiag": (C.c_int, [vp, C.c_int, C.c_int, ip, dp]),
        "qb_batch_clear_history": (C.c_int, [vp]),
        "qb_batch_status": (C.c_int, [vp, C.c_int, ip]),
        "qb_batch_get_tuning": (C.c_int, [vp, C.c_void_p]),
        "qb_batch_set_tuning": (C.c_int, [vp, C.c_void_p]),
        "qb_batch_autotune": (C.c_int, [vp, C.c_int, C.c_void_p]),
        "qb_batch_set_profiling": (C.c_int, [vp, C.c_int]),
        "qb_batch_profile": (C.c_int, [vp, C.c_char_p, C.c_size_t, dp, C.POINTER(C.c_longlong),
                                       C.c_int, ip]),
        "qb_batch_workload": (C.c_int, [vp, dp, C.c_int]),
        "qb_batch_destroy": (None, [vp]),
        "qb_write_re": (C.c_int, [C.c_char_p, C.c_int, dp, dp, C.c_int, fp]),
        "qb_write_re_box": (C.c_int, [C.c_char_p, C.c_int, dp, dp, C.c_int, fp, dp]),
        "qb_append_en": (C.c_int, [C.c_char_p, C.c_int, dp]),
        "qb_append_en_offd": (C.c_int, [C.c_char_p, C.c_int, dp, C.c_int, ip, dp]),
        "qb_fep_analyze": (C.c_int, [dp, ip, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
        "qb_batch_fep": (C.c_int, [vp, ip, C.c_int, C.c_void_p, C.c_void_p]),
        "qb_mlp_forward": (C.c_int, [fp, fp, C.c_int, fp, C.c_int]),
        "qb_mlp_loss_grad": (C.c_int, [fp, fp, fp, C.c_int, fp, fp, C.c_int]),
        "qb_mlp_train": (C.c_int, [fp, fp, fp, C.c_int, C.c_int, C.c_void_p, fp, C.c_int]),
        "qb_mlp_set_wait_limit": (C.c_int, [C.c_longlong]),
        "qb_maxwell": (C.c_int, [C.c_int, C.c_double, C.c_int, dp, dp]),
        "qb_ww_energy_static": (C.c_int, [C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_double, C.c_double,
                                          C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    lib.qb_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != 0:
        raise QBError(rc, last_error())


def exported_symbols() -> list[str]:
    """Names of every function declared in include/*.h."""
    names = []
    for h in sorted(os.listdir(INCLUDE)):
        if h.endswith(".h"):
            src = re.sub(r"/\*.*?\*/", "", open(os.path.join(INCLUDE, h)).read(), flags=re.S)
            names += re.findall(r"^\s*(?:int|void)\s+\**\s*(qb_\w+)\s*\(", src, flags=re.M)
    return names
