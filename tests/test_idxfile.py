"""FastBit index files (.idx) as the library reads them, on the host: the
files under tests/golden/ were written by the reference's own relic::write
and bin::write (tests/golden/make_idx_files.py); their parsed triples must
equal the reference's triples for the same columns.  No device is used."""
import os
import struct

import numpy as np
import pytest

import libfastlib_b200 as L
from conftest import load_golden

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _img(name):
    with open(f"{GOLD}/{name}", "rb") as f:
        return f.read()


def _same_bitmaps(got_offs, got_bms, ref_offs, ref_bms):
    """Bitmap by bitmap; a bitmap the reference's triple leaves empty (no
    bitvector) may be written to a file as an all-zero bitvector."""
    assert len(got_offs) == len(ref_offs)
    for i in range(len(ref_offs) - 1):
        g = got_bms[got_offs[i]:got_offs[i + 1]]
        r = ref_bms[ref_offs[i]:ref_offs[i + 1]]
        if len(r) == 0 and len(g):
            body = g[:-1] if g[-1] == 0 else g[:-2]
            assert all(int(w) & 0xC0000000 == 0x80000000 or int(w) == 0 for w in body), i
            assert g[-1] == 0 or g[-2] == 0, i
        else:
            assert np.array_equal(g, r), i


@pytest.mark.parametrize("suffix", ["", "_o64"])
def test_relic_file_equals_reference_triple(suffix):
    g = load_golden("idxfile_inputs.npz")
    kind, nrows, keys, offs, bms = L.parse_index_file(_img(f"relic_3001{suffix}.idx"))
    assert kind == L.RELIC and nrows == len(g["relic_vals"])
    assert np.array_equal(keys, g["relic_keys"])
    assert np.array_equal(offs, g["relic_offsets"])
    assert np.array_equal(bms, g["relic_bitmaps"])


@pytest.mark.parametrize("suffix", ["", "_o64"])
def test_bin_file_equals_reference_triple(suffix):
    g = load_golden("idxfile_inputs.npz")
    kind, nrows, keys, offs, bms = L.parse_index_file(_img(f"bin_5000{suffix}.idx"))
    assert kind == L.BIN and nrows == len(g["bin_vals"])
    assert np.array_equal(keys, g["bin_keys"])  # minval then maxval
    _same_bitmaps(offs, bms, g["bin_offsets"], g["bin_bitmaps"])


def _relic_image(nrows, keys, bitmaps, osz=4):
    """A relic file laid out as relic::write32/64 do (irelic.cpp:459-642),
    for edge cases the reference's writer does not produce on demand."""
    nobs = len(keys)
    head = b"#IBIS" + bytes([7, osz, 0]) + struct.pack("<III", nrows, nobs, nobs) + b"\0" * 4
    first = 24 + 8 * nobs + osz * (nobs + 1)
    offs, pos = [first], first
    for b in bitmaps:
        pos += 4 * len(b)
        offs.append(pos)
    ot = np.asarray(offs, np.int32 if osz == 4 else np.int64).tobytes()
    body = b"".join(np.asarray(b, np.uint32).tobytes() for b in bitmaps)
    return head + np.asarray(keys, np.float64).tobytes() + ot + body


def test_skipped_bitmap_stays_empty():
    img = _relic_image(62, [1.0, 2.0, 3.0], [[0x80000002, 0], [], [0x40000000, 0x40000000, 0]])
    kind, nrows, keys, offs, bms = L.parse_index_file(img)
    assert kind == L.RELIC and nrows == 62
    assert list(offs) == [0, 2, 2, 5]
    assert list(keys) == [1.0, 2.0, 3.0]


@pytest.mark.parametrize("defect", ["magic", "type", "osz", "truncated", "offset0", "decrease", "odd", "card", "past"])
def test_malformed_files_are_rejected(defect):
    img = bytearray(_relic_image(62, [1.0, 2.0], [[0x80000002, 0], [0x80000002, 0]]))
    first = 24 + 16 + 12
    if defect == "magic":
        img[1] = ord("X")
    elif defect == "type":
        img[5] = 3  # an ambit index: not relic or bin
    elif defect == "osz":
        img[6] = 2
    elif defect == "truncated":
        img = img[:30]
    elif defect == "offset0":
        struct.pack_into("<i", img, 40, first + 4)
    elif defect == "decrease":
        struct.pack_into("<i", img, 44, first - 4)
    elif defect == "odd":
        struct.pack_into("<i", img, 44, first + 6)
    elif defect == "card":
        struct.pack_into("<I", img, 16, 3)
    elif defect == "past":
        struct.pack_into("<i", img, 48, len(img) + 8)
    with pytest.raises(L.WahError) as e:
        L.parse_index_file(bytes(img))
    assert e.value.code == -5  # WAHGPU_EFORMAT


def test_offset_table_checked_before_any_copy():
    """A middle offset past the end of the file, with the last one inside
    it (offsets [first, bytes + 4096, bytes]): the parser rejects the table
    before it copies a bitmap, instead of reading past the image."""
    img = bytearray(_relic_image(62, [1.0, 2.0], [[0x80000002, 0], [0x80000002, 0]]))
    struct.pack_into("<i", img, 44, len(img) + 4096)
    with pytest.raises(L.WahError) as e:
        L.parse_index_file(bytes(img))
    assert e.value.code == -5
