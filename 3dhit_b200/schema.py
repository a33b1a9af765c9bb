"""HDF5 key layout of the files `FieldWriter` and `save_series` write.

The layout is the reference's on-disk format (src/hit3d/schema.py:1-57), so
files written here open in the reference's readers and vice versa:

    grid/{Nx,Ny,Nz,Lx,Ly,Lz[,nu]}        grid metadata, written once
    step_<8-digit step>/{t,<field>}       one group per snapshot
    series/<name>/{t,<field>|values}      one group per recorded series
"""

from __future__ import annotations

__all__ = ["STEP_PREFIX", "step_key", "step_num", "is_step_key", "grid_key", "series_key", "series_field"]

STEP_PREFIX = "step_"
_DIGITS = 8


def step_key(n):
    """Snapshot group of step ``n`` (zero-padded to eight digits)."""
    return STEP_PREFIX + str(int(n)).zfill(_DIGITS)


def is_step_key(key):
    return key.startswith(STEP_PREFIX)


def step_num(key):
    """Step number of a snapshot group name."""
    return int(key[len(STEP_PREFIX):])


def grid_key(name):
    return "grid/" + name


def series_key(name):
    return "series/" + name


def series_field(name, fld):
    return series_key(name) + "/" + fld
