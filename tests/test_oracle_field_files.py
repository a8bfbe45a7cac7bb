"""Oracle of the field file format (pencil-io native MPI-IO v1), pinned to
the reference tests' own fixtures: the header builder of
crates/pencil-io/tests/catalog.rs:57-92 (native_fixture_grid) and the known
payload of crates/pencil-io/tests/mpi_io.rs:105-125 (a [4, 5] i32 field with
extra [2] and value e*1000 + x*100 + y starts at byte 152)."""

import numpy as np

import pencil_oracle as po


def native_fixture_grid(grid, code, width):
    """catalog.rs:57-92 restated: n = 2, extra [3, 2], global [4, 5], zero payload."""
    n, er = 2, 2
    glob, extra, perm = [4, 5], [3, 2], [0, 1]
    hlen = 96 + (n + er + len(grid) + n) * 8
    payload = 4 * 5 * 3 * 2 * width
    h = bytearray(96)
    h[:8] = b"PENCILIO"
    for p, x in [(8, 1), (16, hlen), (24, 0x434F_4D4D_4954_5445), (32, n), (40, code), (48, width), (56, er),
                 (64, hlen), (72, payload), (80, len(grid)), (88, 0)]:
        h[p:p + 8] = x.to_bytes(8, "little")
    for x in glob + extra + list(grid) + perm:
        h += x.to_bytes(8, "little")
    return bytes(h) + bytes(payload)


def test_header_matches_the_reference_fixture_builder():
    for grid in ([2, 1], [1, 3], [2]):
        for dt, (code, width) in [(np.float32, (9, 4)), (np.complex128, (12, 16)), (np.int16, (3, 2))]:
            glob = np.zeros((3, 2, 4, 5), dtype=dt)
            assert po.field_file_bytes(glob, (3, 2), grid, (0, 1)) == native_fixture_grid(grid, code, width)


def test_known_payload_offset_and_values():
    e, x, y = np.indices((2, 4, 5))
    glob = (e * 1000 + x * 100 + y).astype(np.int32)
    data = po.field_file_bytes(glob, (2,), (2, 2), (0, 1))
    assert data[:8] == b"PENCILIO"
    assert data[24:32] == (0x434F_4D4D_4954_5445).to_bytes(8, "little")
    expected = b"".join(int(v).to_bytes(4, "little", signed=True)
                        for e0 in range(2) for x0 in range(4) for y0 in range(5)
                        for v in [e0 * 1000 + x0 * 100 + y0])
    assert data[152:] == expected
