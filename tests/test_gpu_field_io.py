"""Field files written and read by the library (pb_field_write /
pb_field_read, pencil-io's native MPI-IO format v1) against the oracle's
byte-exact restatement: every scalar width (the GPU layout change for
4/8/16-byte elements, the host one for 1/2-byte elements), writer and reader
layouts that differ, exclusive creation, and reads that must fail without
touching the destination (incomplete file, wrong type, wrong shape)."""

import numpy as np
import pytest

import pencil_oracle as po
from pb_testutil import oracle_pencil

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402
from pencil_b200 import fields  # noqa: E402

TORCH = {np.int8: torch.int8, np.int16: torch.int16, np.int32: torch.int32, np.uint64: torch.uint64,
         np.float32: torch.float32, np.float64: torch.float64, np.complex64: torch.complex64,
         np.complex128: torch.complex128}


def to_device(pen, glob, extra_shape):
    n = int(np.prod(extra_shape)) if extra_shape else 1
    flat = po.flat_concat(po.scatter(oracle_pencil(pen), glob.reshape((n,) + pen.global_shape), (n,)))
    t = torch.from_numpy(np.ascontiguousarray(flat).view(np.uint8).copy()).cuda().view(TORCH[glob.dtype.type])
    return fields.PencilArray(pen, t, extra_shape)


@pytest.mark.parametrize("dtype", [np.int8, np.int16, np.int32, np.uint64, np.float32, np.float64, np.complex64,
                                   np.complex128])
def test_write_matches_the_format_and_reads_into_another_layout(dtype, tmp_path):
    rng = np.random.default_rng(7)
    shape, extra = (9, 10, 7), (2, 3)
    writer = pb.Pencil(pb.MpiTopology((2, 3)), shape, (0, 1), (2, 0, 1))
    reader = pb.Pencil(pb.MpiTopology((3, 1)), shape, (1, 2), (0, 1, 2))
    if np.issubdtype(dtype, np.integer):
        glob = rng.integers(0, 100, size=extra + shape).astype(dtype)
    elif np.issubdtype(dtype, np.complexfloating):
        glob = (rng.standard_normal(extra + shape) + 1j * rng.standard_normal(extra + shape)).astype(dtype)
    else:
        glob = rng.standard_normal(extra + shape).astype(dtype)
    src = to_device(writer, glob, extra)
    path = tmp_path / "field.pio"
    fields.write_field(path, src)
    assert path.read_bytes() == po.field_file_bytes(glob, extra, (2, 3), (2, 0, 1))
    dst = fields.PencilArray(reader, torch.zeros_like(to_device(reader, glob, extra).data), extra)
    fields.read_field(path, dst)
    assert torch.equal(dst.data, to_device(reader, glob, extra).data)
    # exclusive creation: an existing file is not overwritten
    before = path.read_bytes()
    with pytest.raises(pb.PencilError) as err:
        fields.write_field(path, src)
    assert err.value.status == "Io" and path.read_bytes() == before


def test_failed_reads_leave_the_destination_unchanged(tmp_path):
    shape = (6, 5, 4)
    pen = pb.Pencil(pb.MpiTopology((2, 2)), shape, (0, 1))
    glob = np.arange(np.prod(shape), dtype=np.float32).reshape(shape)
    path = tmp_path / "ok.pio"
    fields.write_field(path, to_device(pen, glob, ()))
    dst = fields.PencilArray(pen, torch.full((pen.total(),), 7.0, device="cuda"))
    incomplete = tmp_path / "incomplete.pio"
    incomplete.write_bytes(po.field_file_bytes(glob, (), (2, 2), (0, 1, 2), committed=False))
    for bad, kind in ((incomplete, pb.PencilError), (tmp_path / "missing.pio", pb.PencilError)):
        with pytest.raises(kind):
            fields.read_field(bad, dst)
        assert torch.all(dst.data == 7.0)
    wrong_type = fields.PencilArray(pen, torch.full((pen.total(),), 7.0, dtype=torch.float64, device="cuda"))
    with pytest.raises(pb.PencilError) as err:
        fields.read_field(path, wrong_type)
    assert err.value.status == "ShapeMismatch" and torch.all(wrong_type.data == 7.0)
    other = pb.Pencil(pb.MpiTopology((2, 2)), (6, 5, 5), (0, 1))
    wrong_shape = fields.PencilArray(other, torch.full((other.total(),), 7.0, device="cuda"))
    with pytest.raises(pb.PencilError):
        fields.read_field(path, wrong_shape)
    assert torch.all(wrong_shape.data == 7.0)
    truncated = tmp_path / "truncated.pio"
    truncated.write_bytes(path.read_bytes()[:-4])
    with pytest.raises(pb.PencilError):
        fields.read_field(truncated, dst)
    assert torch.all(dst.data == 7.0)
    fields.read_field(path, dst)
    assert torch.equal(dst.data, to_device(pen, glob, ()).data)
