"""The schema-v1 potential archive (src/ptyrodactyl/inout/hdf5.py:1-668).

``save_to_h5(carrier, path)`` / ``load_from_h5(path)`` write and read the reference's
versioned layout: the root carries ``schema_version`` = 1 and the carrier node's
``_node_kind`` = "pytree", ``_pytree_type`` and ``_static_metadata_json``
attributes; each dynamic field is a child dataset (numeric arrays of at least 1 MiB
gzip level 4 with byte shuffling) or a tagged group (``none``, ``json``, ``list``,
``tuple``, ``dict`` with ``_num_items`` / ``_dict_keys_json``); static metadata is
JSON with tagged complex numbers, tuples and mappings. Loading validates the version,
node kinds, carrier type, field set and lengths and rebuilds the carrier through its
factory, so the factory's checks run on every load.

The file format is HDF5 through the h5py API, as in the reference (``h5py.File``,
``create_group``, ``create_dataset``, ``attrs``). ``backend`` selects that API: by
default the ``h5py`` module, imported on first use (a clear ``ImportError`` when it
is absent); any object with the same ``File`` / ``Dataset`` interface works.

Registered carriers: ``PotentialSlices`` (dynamic fields ``slices``,
``slice_thickness``, ``calib``). The reference's schema also registers
``Potential3D``, a volumetric carrier of solvers outside this engine; such archives
are reported as an unknown PyTree type. This build's ``PotentialSlices`` holds float32
slices, so a float64 archive loads rounded to float32.
"""

from __future__ import annotations

import json
from dataclasses import dataclass
from pathlib import Path
from typing import Any, Callable, Dict, Tuple

import numpy as np

from .types import PotentialSlices, create_potential_slices

_ATTR_DICT_KEYS = "_dict_keys_json"
_ATTR_JSON_VALUE = "_json_value"
_ATTR_LENGTH = "_num_items"
_ATTR_NODE_KIND = "_node_kind"
_ATTR_PYTREE_TYPE = "_pytree_type"
_ATTR_SCHEMA_VERSION = "schema_version"
_ATTR_STATIC_METADATA = "_static_metadata_json"
_COMPRESSION_THRESHOLD_BYTES = 1 << 20
_JSON_COMPLEX = "complex"
_JSON_DICT = "dict"
_JSON_KIND = "__ptyrodactyl_json_kind__"
_JSON_TUPLE = "tuple"
_KIND_DICT = "dict"
_KIND_JSON = "json"
_KIND_LIST = "list"
_KIND_NONE = "none"
_KIND_PYTREE = "pytree"
_KIND_TUPLE = "tuple"
SCHEMA_VERSION = 1


class HDF5SchemaError(ValueError):
    """An incompatible or malformed potential archive (hdf5.py:68-73)."""


@dataclass(frozen=True)
class _CarrierMeta:
    cls: type
    factory: Callable[..., Any]
    dynamic_fields: Tuple[str, ...]
    static_fields: Tuple[str, ...] = ()


_REGISTRY: Dict[str, _CarrierMeta] = {
    "PotentialSlices": _CarrierMeta(PotentialSlices, create_potential_slices, ("slices", "slice_thickness", "calib")),
}
_REGISTRY_BY_CLASS = {m.cls: m for m in _REGISTRY.values()}


def _backend(backend):
    if backend is not None:
        return backend
    try:
        import h5py
    except ImportError as error:  # the reference depends on h5py as well
        raise ImportError("save_to_h5 / load_from_h5 need the h5py package") from error
    return h5py


# ----------------------------------------------------------------------------- JSON
def _encode_json_value(value: Any) -> Any:
    """hdf5.py:114-181: tuples, mappings and complex scalars through explicit tags."""
    if value is None or isinstance(value, (bool, int, float, str)):
        return value
    if isinstance(value, complex):
        return {_JSON_KIND: _JSON_COMPLEX, "real": value.real, "imag": value.imag}
    if isinstance(value, np.generic):
        return _encode_json_value(value.item())
    if hasattr(value, "shape"):
        arr = _numpy(value)
        if arr.ndim == 0:
            return _encode_json_value(arr.item())
    if isinstance(value, list):
        return [_encode_json_value(v) for v in value]
    if isinstance(value, tuple):
        return {_JSON_KIND: _JSON_TUPLE, "items": [_encode_json_value(v) for v in value]}
    if isinstance(value, dict):
        return {_JSON_KIND: _JSON_DICT, "items": [[_encode_json_value(k), _encode_json_value(v)]
                                                   for k, v in value.items()]}
    raise TypeError(f"Unsupported static metadata type: {type(value).__name__}")


def _decode_json_value(value: Any) -> Any:
    """hdf5.py:184-227."""
    if isinstance(value, list):
        return [_decode_json_value(v) for v in value]
    if not isinstance(value, dict):
        return value
    marker = value.get(_JSON_KIND)
    if marker == _JSON_COMPLEX:
        return complex(value["real"], value["imag"])
    if marker == _JSON_TUPLE:
        return tuple(_decode_json_value(v) for v in value["items"])
    if marker == _JSON_DICT:
        return {_decode_json_value(k): _decode_json_value(v) for k, v in value["items"]}
    raise HDF5SchemaError("Malformed tagged JSON value in HDF5 archive")


def _numpy(value) -> np.ndarray:
    if hasattr(value, "detach"):  # torch tensors, device or host
        return value.detach().cpu().numpy()
    return np.asarray(value)


def _attribute_text(node, name: str) -> str:
    """hdf5.py:230-259."""
    if name not in node.attrs:
        raise HDF5SchemaError(f"Missing required HDF5 attribute: {name}")
    value = node.attrs[name]
    if isinstance(value, bytes):
        return value.decode("utf-8")
    if isinstance(value, str):
        return value
    raise HDF5SchemaError(f"HDF5 attribute {name!r} must be text")


# ----------------------------------------------------------------------------- write
def _write_carrier_node(node, carrier) -> None:
    """hdf5.py:262-298."""
    meta = _REGISTRY_BY_CLASS.get(type(carrier))
    if meta is None:
        raise TypeError(f"Unsupported carrier type for HDF5 schema version 1: {type(carrier).__name__}")
    node.attrs[_ATTR_NODE_KIND] = _KIND_PYTREE
    node.attrs[_ATTR_PYTREE_TYPE] = type(carrier).__name__
    static = {f: getattr(carrier, f) for f in meta.static_fields}
    node.attrs[_ATTR_STATIC_METADATA] = json.dumps(_encode_json_value(static))
    for f in meta.dynamic_fields:
        value = getattr(carrier, f)
        if isinstance(value, (int, float)) and not isinstance(value, bool):
            # the reference's carrier fields are arrays: scalars are 0-d float64 datasets
            value = np.asarray(value, dtype=np.float64)
        _write_value(node, f, value)


def _write_value(parent, name: str, value) -> None:
    """hdf5.py:301-378."""
    if type(value) in _REGISTRY_BY_CLASS:
        _write_carrier_node(parent.create_group(name), value)
        return
    if value is None:
        parent.create_group(name).attrs[_ATTR_NODE_KIND] = _KIND_NONE
        return
    if isinstance(value, dict):
        group = parent.create_group(name)
        group.attrs[_ATTR_NODE_KIND] = _KIND_DICT
        group.attrs[_ATTR_LENGTH] = len(value)
        group.attrs[_ATTR_DICT_KEYS] = json.dumps([_encode_json_value(k) for k in value])
        for i, item in enumerate(value.values()):
            _write_value(group, f"item_{i}", item)
        return
    if isinstance(value, (list, tuple)):
        group = parent.create_group(name)
        group.attrs[_ATTR_NODE_KIND] = _KIND_LIST if isinstance(value, list) else _KIND_TUPLE
        group.attrs[_ATTR_LENGTH] = len(value)
        for i, item in enumerate(value):
            _write_value(group, f"item_{i}", item)
        return
    if isinstance(value, (bool, int, float, complex, str)):
        group = parent.create_group(name)
        group.attrs[_ATTR_NODE_KIND] = _KIND_JSON
        group.attrs[_ATTR_JSON_VALUE] = json.dumps(_encode_json_value(value))
        return
    arr = _numpy(value)
    if arr.dtype.kind in {"O", "S", "U", "V"}:
        raise TypeError(f"Unsupported array dtype for HDF5 storage: {arr.dtype}")
    options: Dict[str, Any] = {}
    if arr.ndim > 0 and arr.nbytes >= _COMPRESSION_THRESHOLD_BYTES:
        options = {"compression": "gzip", "compression_opts": 4, "shuffle": True}
    parent.create_dataset(name, data=arr, **options)


# ----------------------------------------------------------------------------- read
def _read_carrier_node(node, h5) -> Any:
    """hdf5.py:381-437."""
    kind = _attribute_text(node, _ATTR_NODE_KIND)
    if kind != _KIND_PYTREE:
        raise HDF5SchemaError(f"Unknown HDF5 node kind: {kind}")
    type_name = _attribute_text(node, _ATTR_PYTREE_TYPE)
    meta = _REGISTRY.get(type_name)
    if meta is None:
        raise HDF5SchemaError(f"Unknown PyTree type: {type_name}")
    expected, actual = set(meta.dynamic_fields), set(node.keys())
    if expected - actual:
        raise HDF5SchemaError(f"Missing required carrier field(s): {', '.join(sorted(expected - actual))}")
    if actual - expected:
        raise HDF5SchemaError(f"Unexpected carrier field(s): {', '.join(sorted(actual - expected))}")
    try:
        static = _decode_json_value(json.loads(_attribute_text(node, _ATTR_STATIC_METADATA)))
    except (KeyError, TypeError, json.JSONDecodeError) as error:
        raise HDF5SchemaError("Malformed static metadata in HDF5 archive") from error
    if not isinstance(static, dict):
        raise HDF5SchemaError("Static carrier metadata must be a mapping")
    if set(static) != set(meta.static_fields):
        raise HDF5SchemaError("Static carrier metadata fields do not match")
    fields = {f: _read_value(node[f], h5) for f in meta.dynamic_fields}
    fields.update(static)
    return meta.factory(**fields)


def _read_length(node) -> int:
    """hdf5.py:440-470."""
    if _ATTR_LENGTH not in node.attrs:
        raise HDF5SchemaError(f"Missing required HDF5 attribute: {_ATTR_LENGTH}")
    raw = node.attrs[_ATTR_LENGTH]
    if isinstance(raw, (bool, np.bool_)) or not isinstance(raw, (int, np.integer)):
        raise HDF5SchemaError("HDF5 container length must be an integer")
    if int(raw) < 0:
        raise HDF5SchemaError("HDF5 container length cannot be negative")
    return int(raw)


def _read_items(node, h5, length: int) -> list:
    items = []
    for i in range(length):
        name = f"item_{i}"
        if name not in node:
            raise HDF5SchemaError(f"Missing HDF5 container item: {name}")
        items.append(_read_value(node[name], h5))
    return items


def _read_value(node, h5) -> Any:
    """hdf5.py:473-546: datasets come back as numpy arrays."""
    if isinstance(node, h5.Dataset):
        return np.asarray(node[()])
    kind = _attribute_text(node, _ATTR_NODE_KIND)
    if kind == _KIND_PYTREE:
        return _read_carrier_node(node, h5)
    if kind == _KIND_NONE:
        return None
    if kind == _KIND_JSON:
        try:
            return _decode_json_value(json.loads(_attribute_text(node, _ATTR_JSON_VALUE)))
        except (KeyError, TypeError, json.JSONDecodeError) as error:
            raise HDF5SchemaError("Malformed JSON value in HDF5 archive") from error
    if kind in (_KIND_LIST, _KIND_TUPLE):
        items = _read_items(node, h5, _read_length(node))
        return items if kind == _KIND_LIST else tuple(items)
    if kind == _KIND_DICT:
        length = _read_length(node)
        try:
            keys = [_decode_json_value(k) for k in json.loads(_attribute_text(node, _ATTR_DICT_KEYS))]
        except (KeyError, TypeError, json.JSONDecodeError) as error:
            raise HDF5SchemaError("Malformed dictionary keys in HDF5 archive") from error
        if len(keys) != length:
            raise HDF5SchemaError("HDF5 dictionary length does not match")
        return dict(zip(keys, _read_items(node, h5, length)))
    raise HDF5SchemaError(f"Unknown HDF5 node kind: {kind}")


def _validate_schema_version(handle) -> None:
    """hdf5.py:549-577."""
    if _ATTR_SCHEMA_VERSION not in handle.attrs:
        raise HDF5SchemaError(f"Missing required HDF5 attribute: {_ATTR_SCHEMA_VERSION}")
    raw = handle.attrs[_ATTR_SCHEMA_VERSION]
    if isinstance(raw, (bool, np.bool_)) or not isinstance(raw, (int, np.integer)):
        raise HDF5SchemaError("HDF5 schema_version must be an integer")
    if int(raw) != SCHEMA_VERSION:
        raise HDF5SchemaError(f"Unsupported HDF5 schema_version {int(raw)}; supported version is {SCHEMA_VERSION}")


# ----------------------------------------------------------------------------- API
def save_to_h5(carrier, path, *, backend=None) -> None:
    """Archive one registered carrier; an existing file is replaced (hdf5.py:580-613)."""
    if type(carrier) not in _REGISTRY_BY_CLASS:
        raise TypeError(f"Unsupported carrier type for HDF5 schema version 1: {type(carrier).__name__}")
    h5 = _backend(backend)
    with h5.File(Path(path), "w") as handle:
        handle.attrs[_ATTR_SCHEMA_VERSION] = SCHEMA_VERSION
        _write_carrier_node(handle, carrier)


def load_from_h5(path, *, backend=None):
    """Load one registered carrier through its factory (hdf5.py:616-662)."""
    file_path = Path(path)
    if not file_path.exists():
        raise FileNotFoundError(f"HDF5 file not found: {file_path}")
    h5 = _backend(backend)
    try:
        with h5.File(file_path, "r") as handle:
            _validate_schema_version(handle)
            carrier = _read_carrier_node(handle, h5)
    except HDF5SchemaError:
        raise
    except OSError as error:
        raise HDF5SchemaError(f"Failed to open HDF5 archive {file_path}: {error}") from error
    if not isinstance(carrier, tuple(_REGISTRY_BY_CLASS)):
        raise HDF5SchemaError("Archive did not contain a registered scalar-potential carrier")
    return carrier


__all__ = ["HDF5SchemaError", "load_from_h5", "save_to_h5", "SCHEMA_VERSION"]
