"""The C-ABI library loads and exports every function include/gstb.h declares
(no GPU needed: nothing is called)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "gstb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*[\w\s\*]+?\b(gst_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_entry_points():
    names = declared()
    for must in ("gst_graph_create", "gst_groups_set", "gst_query", "gst_query_batch", "gst_query_noalloc",
                 "gst_serve_open", "gst_serve_submit", "gst_serve_poll", "gst_serve_close"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from gpugst_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_without_device():
    from gpugst_b200 import build
    lib = ctypes.CDLL(build.build())
    lib.gst_status_string.restype = ctypes.c_char_p
    assert lib.gst_status_string(0) == b"ok"
    assert lib.gst_status_string(1) == b"no solution"
    assert lib.gst_status_string(11).startswith(b"query workspace")


def _struct_fields(name):
    src = open(os.path.join(ROOT, "include", "gstb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), src, flags=re.S).group(1)
    names = []
    for decl in re.findall(r"\b(?:uint32_t|uint64_t|int32_t|double)\s+([\w\s,]+);", body):
        names += [n.strip() for n in decl.split(",")]
    return names


def test_python_mirrors_match_the_header_structs():
    """engine.py's ctypes structs list the header's fields in the header's
    order (a field added on one side only would shift every later one)."""
    from gpugst_b200 import engine
    assert list(engine.TUNING_FIELDS) == _struct_fields("gst_tuning")
    assert [f[0] for f in engine._ServeInfo._fields_] == _struct_fields("gst_serve_info")
    assert ctypes.sizeof(engine._Tuning) == 4 * len(engine.TUNING_FIELDS)
