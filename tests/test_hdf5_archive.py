"""The schema-v1 potential archive (ptyrodactyl_b200/hdf5.py) against the reference's
own cases (tests/test_ptyrodactyl/test_inout/test_hdf5.py:1-260), run over an
in-memory stand-in for the h5py API (h5py is not installed in this image): the
layout, the compression rule, round trips and every rejection."""

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from ptyrodactyl_b200.hdf5 import HDF5SchemaError, load_from_h5, save_to_h5
from tests import h5_standin as h5


def _sample():
    """The reference's sample carrier (:29-41), its values exact in float32."""
    return pb.create_potential_slices(
        np.array([[[-3.25, 0.0], [1.5, 8.125], [2.0 ** -40, -(2.0 ** 40)]],
                  [[7.75, -1.25], [3.0, 4.5], [-6.0, 9.0]]]), 1.75, 0.125)


def test_round_trip_is_exact_and_versioned(tmp_path):
    path = tmp_path / "potential.h5"
    expected = _sample()
    save_to_h5(expected, path, backend=h5)
    loaded = load_from_h5(path, backend=h5)
    assert isinstance(loaded, pb.PotentialSlices)
    assert torch.equal(loaded.slices, expected.slices)
    assert loaded.slice_thickness == expected.slice_thickness and loaded.calib == expected.calib
    with h5.File(path, "r") as handle:
        assert int(handle.attrs["schema_version"]) == 1
        assert handle.attrs["_node_kind"] == "pytree"
        assert handle.attrs["_pytree_type"] == "PotentialSlices"
        assert set(handle) == {"calib", "slice_thickness", "slices"}
        for name in handle:
            assert isinstance(handle[name], h5.Dataset)
        assert handle["slice_thickness"].dtype == np.float64 and handle["slice_thickness"][()] == 1.75


def test_large_potential_uses_lossless_gzip_compression(tmp_path):
    path = tmp_path / "large.h5"
    values = np.arange(256 * 256 * 8, dtype=np.float32).reshape(256, 256, 8)  # 2 MiB
    expected = pb.create_potential_slices(values, 2.0, 0.25)
    save_to_h5(expected, path, backend=h5)
    with h5.File(path, "r") as handle:
        s = handle["slices"]
        assert s.compression == "gzip" and s.compression_opts == 4 and s.shuffle and s.chunks is not None
        assert handle["slice_thickness"].compression is None and handle["calib"].compression is None
    assert torch.equal(load_from_h5(path, backend=h5).slices, expected.slices)


@pytest.mark.parametrize("attribute,value,message", [
    ("schema_version", "not-an-integer", "schema_version"),
    ("schema_version", 2, "schema_version"),
    ("schema_version", True, "schema_version"),
    ("_pytree_type", "UnknownPotential", "Unknown.*type"),
    ("_pytree_type", "Potential3D", "Unknown.*type"),
    ("_node_kind", "unknown", "Unknown.*kind"),
    ("_static_metadata_json", "{not json", "Malformed static metadata"),
    ("_static_metadata_json", '{"__ptyrodactyl_json_kind__": "dict", "items": [["x", 1]]}', "fields do not match"),
])
def test_unknown_or_malformed_schema_is_rejected(tmp_path, attribute, value, message):
    path = tmp_path / "mutated.h5"
    save_to_h5(_sample(), path, backend=h5)
    with h5.File(path, "r+") as handle:
        handle.attrs[attribute] = value
    with pytest.raises(HDF5SchemaError, match=message):
        load_from_h5(path, backend=h5)


def test_missing_schema_version_and_fields_are_rejected(tmp_path):
    path = tmp_path / "missing.h5"
    save_to_h5(_sample(), path, backend=h5)
    with h5.File(path, "r+") as handle:
        del handle.attrs["schema_version"]
    with pytest.raises(HDF5SchemaError, match="schema_version"):
        load_from_h5(path, backend=h5)
    save_to_h5(_sample(), path, backend=h5)
    with h5.File(path, "r+") as handle:
        del handle._children["calib"]
        handle.create_dataset("extra", data=np.zeros(2))
    with pytest.raises(HDF5SchemaError, match="Missing required carrier field"):
        load_from_h5(path, backend=h5)


def test_reload_runs_the_factory_validation(tmp_path):
    path = tmp_path / "invalid.h5"
    save_to_h5(_sample(), path, backend=h5)
    with h5.File(path, "r+") as handle:
        handle["slice_thickness"][...] = -1.0
    with pytest.raises(ValueError, match="slice_thickness"):
        load_from_h5(path, backend=h5)


def test_unsupported_carriers_files_and_backend(tmp_path):
    with pytest.raises(TypeError, match="Unsupported carrier type"):
        save_to_h5({"slices": 1}, tmp_path / "x.h5", backend=h5)
    with pytest.raises(FileNotFoundError):
        load_from_h5(tmp_path / "absent.h5", backend=h5)
    bad = tmp_path / "garbage.h5"
    bad.write_bytes(b"not an archive")
    with pytest.raises(HDF5SchemaError, match="Failed to open"):
        load_from_h5(bad, backend=h5)
    try:
        import h5py  # noqa: F401
    except ImportError:
        with pytest.raises(ImportError, match="h5py"):
            save_to_h5(_sample(), tmp_path / "y.h5")


def test_node_codec_round_trips_containers_and_tagged_json(tmp_path):
    """The general node codec (hdf5.py:114-546): None, JSON scalars incl. complex,
    lists, tuples, dicts with tuple keys, nested carriers and arrays."""
    from ptyrodactyl_b200 import hdf5 as H
    value = {"a": [1, 2.5, None, "text", 1 + 2j], (1, "k"): (np.arange(3), {"inner": _sample()}), "z": True}
    path = tmp_path / "nodes.h5"
    with h5.File(path, "w") as handle:
        H._write_value(handle, "root", value)
    with h5.File(path, "r") as handle:
        got = H._read_value(handle["root"], h5)
    assert list(got) == ["a", (1, "k"), "z"]
    assert got["a"] == [1, 2.5, None, "text", 1 + 2j] and got["z"] is True
    arr, inner = got[(1, "k")]
    assert np.array_equal(arr, np.arange(3))
    assert torch.equal(inner["inner"].slices, _sample().slices)
    with pytest.raises(TypeError, match="Unsupported array dtype"):
        with h5.File(tmp_path / "bad.h5", "w") as handle:
            H._write_value(handle, "s", np.array(["a", "b"]))
    with pytest.raises(HDF5SchemaError, match="Malformed tagged JSON"):
        H._decode_json_value({"__ptyrodactyl_json_kind__": "weird"})
