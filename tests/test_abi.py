"""CPU tests of the drop-in boundary: the C ABI library loads and exports every
declared entry point, and the Python layer keeps the reference's codecs and
error behaviour without touching a GPU."""

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

import finitevolumegpu_b200 as fv
from finitevolumegpu_b200 import _lib
from finitevolumegpu_b200.Simulator import BoundaryCondition, stepOrderToCodedInt

HEADER = os.path.join(ROOT, "include", "fvgpu.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^FV_API\s+[\w\s\*]+?\b(fv_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in ("fv_sim_create", "fv_sim_simulate", "fv_sim_step", "fv_sim_substep", "fv_sim_download",
              "fv_sim_compute_dt", "fv_context_create", "fv_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    for s in declared_symbols():
        assert hasattr(L, s), s
    assert L.fv_version() >= 100


def test_python_binding_covers_header():
    assert set(declared_symbols()) <= set(_lib._SIGNATURES)


def test_oracle_library_exports():
    from oracle import oracle

    L = oracle.lib()
    for s in ("fvo_substep_f32", "fvo_substep_f64", "fvo_ghost_cells", "fvo_num_vars"):
        assert hasattr(L, s)
    assert L.fvo_ghost_cells(0) == 1 and L.fvo_ghost_cells(6) == 2 and L.fvo_num_vars(7) == 4


def test_boundary_condition_codec():
    T = BoundaryCondition.Type
    bc = BoundaryCondition({"north": T.Periodic, "south": T.Reflective, "east": T.Dirichlet, "west": T.Periodic})
    code = int(bc.asCodedInt())
    assert code == (2 << 24) | (3 << 16) | (0 << 8) | 2
    back = BoundaryCondition.getTypes(code)
    assert back == {"north": T.Periodic, "south": T.Reflective, "east": T.Dirichlet, "west": T.Periodic}
    assert int(BoundaryCondition().asCodedInt()) == 0x03030303


def test_neumann_rejected():
    T = BoundaryCondition.Type
    with pytest.raises(NotImplementedError):
        BoundaryCondition({"north": T.Neumann, "south": T.Reflective, "east": T.Reflective, "west": T.Reflective})


def test_step_order_codec():
    assert int(stepOrderToCodedInt(1, 2)) == (1 << 16) | 2
    assert int(stepOrderToCodedInt(0, 1)) == 1


class _NoGpuContext:
    handle = None
    autotuner = None
    device_name = "none"


@pytest.mark.parametrize("shape", [(10, 9), (13, 13), (12, 10, 1)])
def test_constructor_rejects_bad_shapes(shape):
    a = np.ones(shape, np.float32)
    with pytest.raises(AssertionError):
        fv.KP07_dimsplit.KP07_dimsplit(_NoGpuContext(), a, a, a, 10, 8, 1.0, 1.0, 9.81)


def test_constructor_rejects_wrong_itemsize():
    a = np.ones((8, 10), np.float64)
    with pytest.raises(AssertionError):
        fv.HLL.HLL(_NoGpuContext(), a, a, a, 10, 8, 1.0, 1.0, 9.81)


def test_class_signatures_match_reference():
    import inspect

    sig = inspect.signature(fv.KP07_dimsplit.KP07_dimsplit.__init__)
    assert list(sig.parameters)[1:] == ["context", "h0", "hu0", "hv0", "nx", "ny", "dx", "dy", "g", "theta",
                                        "cfl_scale", "boundary_conditions", "block_width", "block_height"]
    assert sig.parameters["theta"].default == 1.3 and sig.parameters["cfl_scale"].default == 0.9
    sig = inspect.signature(fv.EE2D_KP07_dimsplit.EE2D_KP07_dimsplit.__init__)
    assert list(sig.parameters)[1:11] == ["context", "rho", "rho_u", "rho_v", "E", "nx", "ny", "dx", "dy", "g"]
    assert sig.parameters["block_height"].default == 8
    assert inspect.signature(fv.HLL2.HLL2.__init__).parameters["theta"].default == 1.8
    assert inspect.signature(fv.KP07.KP07.__init__).parameters["order"].default == 2
    for name in ("LxF", "FORCE", "HLL", "WAF"):
        assert "theta" not in inspect.signature(fv.SCHEMES[name].__init__).parameters


def test_no_cpu_fallback():
    """Without a usable GPU the context raises; nothing silently computes on the host."""
    import subprocess
    import sys

    code = ("import sys; sys.path.insert(0, %r)\n"
            "from finitevolumegpu_b200 import CudaContext\n"
            "try:\n    CudaContext.CudaContext()\nexcept Exception as e:\n    print('raised', type(e).__name__)\n"
            "else:\n    print('ok')\n" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=dict(
        os.environ, CUDA_VISIBLE_DEVICES=""))
    assert "raised" in out.stdout, out.stdout + out.stderr


def test_shape_checks_survive_python_O():
    """The checks that guard host buffer sizes are not assert statements: under
    ``python -O`` a mismatched variable still raises before any C call."""
    import subprocess
    import sys

    code = ("import sys; sys.path.insert(0, %r)\n"
            "import numpy as np\n"
            "import finitevolumegpu_b200 as fv\n"
            "class C:\n    handle = None\n    autotuner = None\n    device_name = 'none'\n"
            "a = np.ones((8, 10), np.float32); b = np.ones((8, 9), np.float32)\n"
            "try:\n    fv.KP07_dimsplit.KP07_dimsplit(C(), a, b, a, 10, 8, 1.0, 1.0, 9.81)\n"
            "except AssertionError as e:\n    print('raised', e)\n"
            "else:\n    print('ok')\n" % ROOT)
    out = subprocess.run([sys.executable, "-O", "-c", code], capture_output=True, text=True)
    assert "raised" in out.stdout, out.stdout + out.stderr


@pytest.mark.parametrize("n_vars,shape", [(2, (8, 10)), (3, (8, 9))])
def test_batch_add_rejects_bad_inputs(n_vars, shape):
    from finitevolumegpu_b200.batch import Batch

    b = Batch.__new__(Batch)  # no device: add() must refuse before reaching the library
    b.scheme, b.nv, b.gc, b._h, b.shapes = "KP07_dimsplit", 3, 2, None, {}
    good = np.ones((8, 10), np.float32)
    arrays = [good] * (n_vars - 1) + [np.ones(shape, np.float32)]
    with pytest.raises(AssertionError):
        b.add(arrays, 10, 8, 1.0, 1.0, 1.0)


def _header_prototypes():
    """{name: (return type, [parameter types])} of every FV_API function."""
    src = re.sub(r"/\*.*?\*/", " ", open(HEADER).read(), flags=re.S)
    protos = {}
    for ret, name, params in re.findall(r"^FV_API\s+([\w\s\*]+?)\s*\b(fv_\w+)\s*\((.*?)\);", src, flags=re.M | re.S):
        types = []
        for p in params.split(","):
            p = " ".join(p.split())
            if p in ("", "void"):
                continue
            ptr = p.count("*")
            words = [w for w in re.findall(r"[A-Za-z_]\w*", p) if w != "const"]
            base = " ".join(words[:-1]) if len(words) > 1 else words[0]  # drop the parameter name
            types.append("ptr" if ptr else base)
        protos[name] = (("ptr" if "*" in ret else " ".join(ret.split())), types)
    return protos


def _kind(ctype):
    scalars = {ctypes.c_int: "int", ctypes.c_float: "float", ctypes.c_double: "double",
               ctypes.c_longlong: "long long", ctypes.c_size_t: "size_t"}
    if ctype in scalars:
        return scalars[ctype]
    if ctype in (ctypes.c_void_p, ctypes.c_char_p) or hasattr(ctype, "_type_") and issubclass(
            ctype, ctypes._Pointer):
        return "ptr"
    return repr(ctype)


def test_python_argtypes_match_header_prototypes():
    """Every ctypes declaration passes as many arguments, of the same kinds, as
    the C prototype takes: a mismatch would pass garbage through the ABI."""
    protos = _header_prototypes()
    assert len(protos) == len(declared_symbols())
    for name, (ret, params) in protos.items():
        args, res = _lib._SIGNATURES[name]
        assert [_kind(a) for a in args] == params, name
        assert _kind(res) == ret, name


def test_python_constants_and_params_match_header():
    """Status codes, scheme ids and the fv_params layout restated in _lib.py
    are the header's."""
    src = re.sub(r"/\*.*?\*/", " ", open(HEADER).read(), flags=re.S)
    codes = dict((k, int(v)) for k, v in re.findall(r"#define (FV_(?:OK|ERR_\w+))\s+(\d+)", src))
    assert codes == {k: getattr(_lib, k) for k in codes} and len(codes) == 6
    enum = dict((k, int(v)) for k, v in re.findall(r"FV_(\w+) = (\d+)", src))
    ids = {k.upper(): v for k, v in _lib.SCHEME_IDS.items()}
    assert enum == ids
    body = re.search(r"typedef struct fv_params \{(.*?)\} fv_params;", src, re.S).group(1)
    fields = re.findall(r"(float|int)\s+(\w+);", body)
    ctype = {"float": ctypes.c_float, "int": ctypes.c_int}
    assert [(n, ctype[t]) for t, n in fields] == list(_lib.fv_params._fields_)


def test_null_handles_are_rejected_before_any_cuda_call():
    """Every entry point that takes a simulation or batch handle answers a null
    handle with FV_ERR_INVALID and an error message (checked before any CUDA call, so
    this runs without a GPU); destroying a null handle is a no-op."""
    L = _lib.lib()
    zero = {ctypes.c_int: 0, ctypes.c_float: 0.0, ctypes.c_double: 0.0, ctypes.c_longlong: 0}
    names = [n for n in _lib._SIGNATURES if n.startswith(("fv_sim_", "fv_batch_"))
             and not n.endswith(("_create", "_destroy"))]
    assert len(names) >= 30
    for name in names:
        args, _ = _lib._SIGNATURES[name]
        call = [zero.get(a) for a in args]  # pointers (and the handle) are NULL
        rc = getattr(L, name)(*call)
        assert rc == _lib.FV_ERR_INVALID, (name, rc)
        assert L.fv_last_error().decode(), name  # a message for fv_last_error
    assert L.fv_sim_destroy(None) == _lib.FV_OK and L.fv_batch_destroy(None) == _lib.FV_OK
    assert L.fv_context_destroy(None) == _lib.FV_OK
    assert L.fv_context_device_name(None, None, 0) == _lib.FV_ERR_INVALID


def test_noalloc_argument_checks_come_before_any_cuda_call():
    """The allocation-free substep refuses unknown wall codes, Neumann walls and
    output planes that overlap an input plane or each other before it touches
    the GPU (the addresses below are never dereferenced)."""
    L = _lib.lib()
    FP = _lib._FP
    nx, ny = 100, 50
    pitch = nx + 8
    plane = (ny + 4) * pitch * 4

    def planes(base):
        return (FP * 3)(*[ctypes.cast(base + k * plane, FP) for k in range(3)])

    ins, outs = planes(1 << 32), planes((1 << 32) + 3 * plane)

    def call(i, o, bc=0x03030303):
        return L.fv_kp07_dimsplit_substep_noalloc(i, o, pitch, nx, ny, 1.0, 1.0, 0.01, 9.81, 1.3, 0, bc, None, None)

    for bc in (0x03030304, 0x0F000000, 0x03030313):
        assert call(ins, outs, bc) == _lib.FV_ERR_INVALID, hex(bc)
    assert call(ins, outs, 0x01030303) == _lib.FV_ERR_UNSUPPORTED
    assert call(ins, ins) == _lib.FV_ERR_INVALID
    assert "overlap" in L.fv_last_error().decode()
    shifted = (FP * 3)(*[ctypes.cast((1 << 32) + 3 * plane - 16, FP), outs[1], outs[2]])
    assert call(ins, shifted) == _lib.FV_ERR_INVALID  # last 16 bytes of the third input plane
    same = (FP * 3)(outs[0], outs[0], outs[2])
    assert call(ins, same) == _lib.FV_ERR_INVALID
