"""Loader for the reference's own numba hot-path modules (test infrastructure).

This module is ORACLE / TEST INFRASTRUCTURE. It is only ever used in a
container where the EMerge source tree is present, to generate the golden
fixtures committed under ``tests/golden/`` (see ``tests/golden/make_golden.py``).
Nothing in the product package, the GPU tests, ``smoke()`` or ``bench.py``
imports it.

The reference package ``emerge`` cannot be imported normally here because its
top-level ``__init__`` pulls in gmsh / emsutil / pyvista. Its hot-path modules
only depend on numpy, numba, scipy and loguru, so we register empty parent
packages whose ``__path__`` points into the source tree and import the leaf
modules directly:

* ``emerge._emerge.physics.microwave.assembly.curlcurl``
  (``_matrix_builder`` curlcurl.py:387-456, ``ned2_tet_stiff_mass`` :285-380,
  ``tet_coefficients`` :127-214)
* ``emerge._emerge.mth.csc_cast`` (``CSCMapping`` :29-63,
  ``precompute_csc_pattern`` :65-160, ``scatter_to_csc_c16`` :162-177)
* ``emerge._emerge.mth.optimized`` (``local_mapping`` :262-296, ``matinv`` :315-357)
* ``emerge._emerge.physics.microwave.assembly.robinbc`` (``ned2_tri_stiff``
  :316-378, ``compute_bc_entries`` :381-402)
* ``emerge._emerge.physics.heatconduction.assembly.grad`` (``leg2_tet_stiff``
  :199-260, ``leg2_tet_mass`` :263-330, the COO builders :333-400)
* ``emerge._emerge.compiled.base.interp`` (``ned2_tet_interp`` :286-387) and
  ``emerge._emerge.mth.integrals`` (``surface_integral`` :64-103)
"""
from __future__ import annotations

import importlib
import os
import sys
import tempfile
import types

DEFAULT_REF_ROOT = "/root/reference"


def _pkg(name: str, path: str | None) -> types.ModuleType:
    mod = types.ModuleType(name)
    mod.__path__ = [path] if path else []
    sys.modules[name] = mod
    return mod


def load_reference(ref_root: str = DEFAULT_REF_ROOT):
    """Import the reference hot-path modules; returns a namespace with
    ``curlcurl``, ``csc_cast``, ``optimized`` and ``ccbf``."""
    src = os.path.join(ref_root, "src", "emerge")
    if not os.path.isdir(src):
        raise FileNotFoundError(f"reference source tree not found under {ref_root}")
    # numba wants a writable cache dir; the reference tree is read-only.
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "emerge_ref_numba_cache"))
    em = os.path.join(src, "_emerge")
    if "emerge._emerge.physics.microwave.assembly.curlcurl" not in sys.modules:
        _pkg("emerge", src)
        _pkg("emerge._emerge", em)
        _pkg("emerge._emerge.mth", os.path.join(em, "mth"))
        _pkg("emerge._emerge.compiled", os.path.join(em, "compiled"))
        _pkg("emerge._emerge.physics", os.path.join(em, "physics"))
        _pkg("emerge._emerge.physics.microwave", os.path.join(em, "physics", "microwave"))
        _pkg("emerge._emerge.physics.microwave.assembly",
             os.path.join(em, "physics", "microwave", "assembly"))
        elements = _pkg("emerge._emerge.elements", None)
        elements.Nedelec2 = object  # only used as a type hint by curlcurl.py:21
    ns = types.SimpleNamespace()
    ns.curlcurl = importlib.import_module("emerge._emerge.physics.microwave.assembly.curlcurl")
    ns.csc_cast = importlib.import_module("emerge._emerge.mth.csc_cast")
    ns.optimized = importlib.import_module("emerge._emerge.mth.optimized")
    ns.ccbf = importlib.import_module("emerge._emerge.compiled.ccbf")
    # Robin boundary term (robinbc.py); imports cleanly with the stubs above
    ns.robinbc = importlib.import_module("emerge._emerge.physics.microwave.assembly.robinbc")
    # second-order absorbing boundary correction (robin_abc_order2.py)
    ns.abc2 = importlib.import_module("emerge._emerge.physics.microwave.assembly.robin_abc_order2")
    # post-processing: field interpolation and surface integrals
    if "emerge._emerge.compiled.base" not in sys.modules:
        _pkg("emerge._emerge.compiled.base", os.path.join(em, "compiled", "base"))
    ns.interp = importlib.import_module("emerge._emerge.compiled.base.interp")
    # heat conduction (grad.py imports Legrange2 as a type hint only)
    if "emerge._emerge.physics.heatconduction.assembly.grad" not in sys.modules:
        _pkg("emerge._emerge.physics.heatconduction", os.path.join(em, "physics", "heatconduction"))
        _pkg("emerge._emerge.physics.heatconduction.assembly",
             os.path.join(em, "physics", "heatconduction", "assembly"))
        leg2 = types.ModuleType("emerge._emerge.elements.leg2")
        leg2.Legrange2 = object
        sys.modules["emerge._emerge.elements.leg2"] = leg2
    ns.heat = importlib.import_module("emerge._emerge.physics.heatconduction.assembly.grad")
    ns.integrals = importlib.import_module("emerge._emerge.mth.integrals")
    return ns


def _module_from_file(name: str, path: str) -> types.ModuleType:
    import importlib.util
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_nedelec2(ref_root: str = DEFAULT_REF_ROOT):
    """The reference's Nedelec-2 basis class (``elements/nedelec2.py``, with
    ``femdata.FEMBasis`` and ``dofsets``) for generating the partitioned-field
    (ThinConductor) fixture. Its imports of the mesh class, the ``emsutil``
    save mixin and the compiled interpolation library are stubbed: the
    constructor, ``partition_dof``, ``empty_tri_rowcol`` and ``generate_csc``
    only read the mesh object they are given. Call after ``load_reference``."""
    em = os.path.join(ref_root, "src", "emerge", "_emerge")
    if "emsutil" not in sys.modules:
        try:
            importlib.import_module("emsutil")
        except ImportError:
            stub = types.ModuleType("emsutil")
            stub.Saveable = object
            sys.modules["emsutil"] = stub
    if "emerge._emerge.mesh3d" not in sys.modules:
        m3 = types.ModuleType("emerge._emerge.mesh3d")
        m3.Mesh3D = object  # a type hint only
        sys.modules["emerge._emerge.mesh3d"] = m3
    comp = sys.modules["emerge._emerge.compiled"]
    if not hasattr(comp, "MATHLIB"):
        comp.MATHLIB = None  # the interpolators are not called
    el = os.path.join(em, "elements")
    ns = types.SimpleNamespace()
    ns.dofsets = _module_from_file("emerge._emerge.elements.dofsets", os.path.join(el, "dofsets.py"))
    ns.femdata = _module_from_file("emerge._emerge.elements.femdata", os.path.join(el, "femdata.py"))
    ns.nedelec2 = _module_from_file("emerge._emerge.elements.nedelec2", os.path.join(el, "nedelec2.py"))
    return ns
