"""HDF5 filter 61197 on the GPU codec (python/pywaltz/hdf5.py of the
reference project).

``plugin_path()`` is the directory holding ``libwaltz_h5z.so``, an HDF5
filter plugin with the reference plugin's client data and chunk archives;
``filter_values`` gives that client data. ``enable_filter`` and
``create_dataset`` need h5py, imported when they are called.
"""

import operator
import os
import struct
import sys
from contextlib import closing
from pathlib import Path

import waltz_b200

from .codec import _bound, _geometry

FILTER_ID = 61197


def plugin_path():
    """Directory of the filter plugin library."""
    return Path(waltz_b200.__file__).resolve().with_name("plugins")


def filter_values(chunks, dtype, abs_error):
    """The filter's six client-data words for (z,y,x) or (y,x) chunks:
    nx, ny, nz, sample width, then the bound's double as two 32-bit words."""
    dims, dtype = _geometry(tuple(chunks)[-3:], dtype)
    lo, hi = struct.unpack("<II", struct.pack("<d", _bound(abs_error)))
    return (*dims, dtype.itemsize, lo, hi)


def enable_filter():
    """Make HDF5 find the plugin (prepends plugin_path() to its search path)."""
    import h5py
    path = os.fsencode(plugin_path())
    pl = h5py.h5pl
    if os.path.isdir(path) and path not in (pl.get(i) for i in range(pl.size())):
        pl.prepend(path)
    if not h5py.h5z.filter_avail(FILTER_ID):
        raise RuntimeError("Waltz HDF5 filter plugin not found: run `python -m waltz_b200.build`")


def create_dataset(group, name, *, shape, chunks, dtype, abs_error):
    """Create an empty fixed-size chunked dataset with the mandatory filter.

    2-D / 3-D chunks use (y,x) / (z,y,x); a 4-D stack (n,z,y,x) has one
    sample per chunk along n. Edge chunks use HDF5 zero fill."""
    import h5py
    shape = tuple(map(operator.index, shape))
    chunks = tuple(map(operator.index, chunks))
    if len(shape) not in (2, 3, 4) or len(chunks) != len(shape):
        raise ValueError("shape and chunks must have the same rank (2, 3 or 4)")
    if any(c <= 0 or c > s for c, s in zip(chunks, shape)):
        raise ValueError("require 0 < chunk extent <= dataset extent on each axis")
    if len(chunks) == 4 and chunks[0] != 1:
        raise ValueError("4-D data must use a leading chunk extent of 1")
    if sys.byteorder != "little":
        raise ValueError("the Waltz HDF5 filter requires a little-endian host")
    values = filter_values(chunks, dtype, abs_error)
    enable_filter()
    with closing(h5py.h5p.create(h5py.h5p.DATASET_CREATE)) as dcpl:
        dcpl.set_chunk(chunks)
        dcpl.set_filter(FILTER_ID, h5py.h5z.FLAG_MANDATORY, values)
        with closing(h5py.h5s.create_simple(shape)) as space, \
                closing(h5py.h5t.py_create(__import__("numpy").dtype(dtype))) as tid:
            did = h5py.h5d.create(group.id, name.encode("utf-8"), tid, space, dcpl=dcpl)
    return h5py.Dataset(did)
