"""Checkpoint / restart of long evolutions (the `_temp.mat` restart files of
examples/rydberg_pollution_density_matrix_gpu_restart.jl:151-189, writer `write_data_file`
:238-266).

Two containers, chosen by the file name.  ``*.mat``: a MAT v5 file (scipy.io), readable by
MATLAB, MAT.jl and scipy, with the reference writer's variable names; an MPS (a device
``MPS`` or a list of host site arrays, the reference's ``collect.(rho)``) is a cell array of
complex ``[chiL, d, chiR]`` sites, as MAT.jl writes a Vector of arrays (the reference's own
files are MAT v7.3, an HDF5 layout no library here writes).  Anything else: NumPy's ``.npz``
with each MPS site stored as ``<name>/<k>``.  MPS fields are restored as device ``MPS``
objects (or host sites).  A write goes to ``<file>.tmp`` first and is renamed into place, so
an interrupted write never replaces the previous checkpoint.
"""
import json
import os

import numpy as np

_MPS_KEY = "__mps__"
# MAT variable holding the exact shape of every non-MPS field (JSON), so that a size-1 array or a
# 1 x n matrix reads back with the shape it was written with (MAT stores everything as >= 2-d)
_MAT_SHAPES = "mpsb_field_shapes"


def _mps_sites(v):
    if hasattr(v, "sites") and hasattr(v, "dims"):          # device MPS
        return v.sites()
    if isinstance(v, (list, tuple)) and v and all(isinstance(a, np.ndarray) and a.ndim == 3 for a in v):
        return list(v)
    return None


def _is_mat(filename):
    return filename.lower().endswith(".mat")


def write_data_file(filename, fields):
    """Write ``fields`` (name -> scalar / array / MPS / list of site arrays) to ``filename``."""
    if _is_mat(filename):
        return _write_mat(filename, fields)
    arrays, mps_names = {}, []
    for name, v in fields.items():
        if "/" in name or name == _MPS_KEY:
            raise ValueError("field name %r is reserved" % name)
        sites = _mps_sites(v)
        if sites is not None:
            mps_names.append(name)
            for k, a in enumerate(sites):
                arrays["%s/%d" % (name, k)] = np.asarray(a, dtype=np.complex128)
        else:
            arrays[name] = np.asarray(v)
    arrays[_MPS_KEY] = np.frombuffer(json.dumps(mps_names).encode(), dtype=np.uint8)
    tmp = filename + ".tmp"
    with open(tmp, "wb") as f:
        np.savez(f, **arrays)
    os.replace(tmp, filename)


def _write_mat(filename, fields):
    import scipy.io
    out, shapes = {}, {}
    for name, v in fields.items():
        if not name.isidentifier() or name == _MAT_SHAPES:
            raise ValueError("field name %r is not a MAT variable name" % name)
        sites = _mps_sites(v)
        if sites is not None:
            cell = np.empty((len(sites), 1), dtype=object)   # a column cell array, as MAT.jl writes
            for k, a in enumerate(sites):
                cell[k, 0] = np.asarray(a, dtype=np.complex128)
            out[name] = cell
        else:
            out[name] = np.asarray(v)
            if out[name].dtype.kind != "U":
                shapes[name] = list(out[name].shape)
    out[_MAT_SHAPES] = json.dumps(shapes)
    tmp = filename + ".tmp"
    with open(tmp, "wb") as f:
        scipy.io.savemat(f, out, format="5", do_compression=False, oned_as="row")
    os.replace(tmp, filename)


def _read_mat(filename):
    import scipy.io
    raw = scipy.io.loadmat(filename, squeeze_me=False, chars_as_strings=True)
    shapes = json.loads(str(raw.pop(_MAT_SHAPES)[0])) if _MAT_SHAPES in raw else None
    out, mps = {}, {}
    for name, a in raw.items():
        if name.startswith("__"):
            continue
        if a.dtype == object:                                  # a cell array: an MPS
            mps[name] = [np.asarray(c, dtype=np.complex128).reshape(c.shape + (1,) * (3 - c.ndim))
                         for c in a.ravel(order="F")]
        elif a.dtype.kind == "U":
            out[name] = str(a[0]) if a.size else ""
        elif shapes is not None and name in shapes:
            # only the 0-d / 1-d fields changed shape on the way out (to 1 x 1 / 1 x n)
            shp = tuple(shapes[name])
            b = a.reshape(shp) if a.size == int(np.prod(shp)) else a
            out[name] = b.item() if b.ndim == 0 else b
        else:
            # a file written elsewhere (the reference's writer): 1 x 1 -> scalar, a 1 x n row -> 1-d
            out[name] = a.reshape(()).item() if a.size == 1 else (a.ravel() if a.ndim == 2 and a.shape[0] == 1 else a)
    return out, mps


def read_data_file(filename, ctx=None, device=True):
    """Read a checkpoint.  MPS fields come back as device ``MPS`` objects on ``ctx`` (the
    default context when None) if ``device``, else as lists of host site arrays.  Every other
    field comes back with the shape it was written with (0-d arrays as Python scalars); in a MAT
    file written elsewhere, 1 x 1 values come back as scalars and 1 x n rows as 1-d arrays."""
    if _is_mat(filename):
        out, mps = _read_mat(filename)
        for name, sites in mps.items():
            if device:
                from .core import MPS
                out[name] = MPS.from_sites(sites, ctx)
            else:
                out[name] = sites
        return out
    out = {}
    with np.load(filename, allow_pickle=False) as z:
        mps_names = json.loads(bytes(z[_MPS_KEY]).decode())
        for name in z.files:
            if name == _MPS_KEY or "/" in name:
                continue
            a = z[name]
            out[name] = a.item() if a.ndim == 0 else a
        for name in mps_names:
            n = sum(1 for f in z.files if f.startswith(name + "/"))
            sites = [z["%s/%d" % (name, k)] for k in range(n)]
            if device:
                from .core import MPS
                out[name] = MPS.from_sites(sites, ctx)
            else:
                out[name] = sites
    return out
