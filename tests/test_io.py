"""Cloud files in the reference's formats, host side (no GPU): the text reader
against the reference's own rd::Samples<float>::loadFromFile, binary files
against numpy."""
import os

import numpy as np
import pytest

import oracle as O
import ridgedetection_b200 as rdb


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_bytes(text.encode())
    return str(p)


def _ref_or_skip():
    if O.ref(False) is None:
        pytest.skip("oracle/_ref not built")


TEXTS = {
    "trailing_space": "".join(f"{a:.7g} {b:.7g} {c:.7g} \n" for a, b, c in
                              np.random.default_rng(1).normal(size=(500, 3))),
    "tabs": "".join(f"{a:.9g}\t{b:.9g}\t\n" for a, b in np.random.default_rng(2).random((300, 2))),
    "no_trailing_space": "".join(f"{a:.6g} {b:.6g} {c:.6g}\n" for a, b, c in
                                 np.random.default_rng(3).normal(size=(200, 3))),
    "ragged_lines": "1 2 3 \n4 5\n6 7 8 9 \n",
}


@pytest.mark.parametrize("name", sorted(TEXTS))
def test_text_reader_matches_reference(tmp_path, name):
    _ref_or_skip()
    path = _write(tmp_path, name + ".txt", TEXTS[name])
    ref = O.ref_load_text(path)
    got = rdb.load_text_cloud(path)
    assert ref is not None
    assert got.shape == ref.shape
    if name == "ragged_lines":  # the reference leaves missing values unset
        assert np.array_equal(got[[0, 2]], ref[[0, 2]])
        assert got[1, 2] == 0.0 and np.array_equal(got[1, :2], ref[1, :2])
    else:
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_text_dimension_rule(tmp_path):
    """Without trailing white space the last value of the first line is not counted."""
    assert rdb.load_text_cloud(_write(tmp_path, "a.txt", "1 2 3\n4 5 6\n")).shape == (2, 2)
    assert rdb.load_text_cloud(_write(tmp_path, "b.txt", "1 2 3 \n4 5 6 \n")).shape == (2, 3)


@pytest.mark.parametrize("text", ["1 2 \n\n3 4 \n", "1 2 \n3 4 "])
def test_text_count_mismatch_is_an_error(tmp_path, text):
    """Blank lines or a last line without a newline: the count of newlines and
    of points differ, which the reference rejects too."""
    path = _write(tmp_path, "bad.txt", text)
    with pytest.raises(rdb.RDError):
        rdb.load_text_cloud(path)
    if O.ref(False) is not None:
        assert O.ref_load_text(path) is None


def test_binary_round_trip_and_short_file(tmp_path):
    P = np.random.default_rng(4).normal(size=(1000, 3)).astype(np.float32)
    path = str(tmp_path / "c.bin")
    rdb.save_binary_cloud(path, P)
    assert os.path.getsize(path) == P.nbytes
    assert np.array_equal(rdb.load_binary_cloud(path, 1000, 3), P)
    assert np.array_equal(rdb.load_binary_cloud(path, 500, 3), P[:500])   # longer file is fine
    P.tofile(str(tmp_path / "d.bin"))
    assert np.array_equal(rdb.load_binary_cloud(str(tmp_path / "d.bin"), 1000, 3), P)
    with pytest.raises(rdb.RDError):
        rdb.load_binary_cloud(path, 1001, 3)
    with pytest.raises(rdb.RDError):
        rdb.load_binary_cloud(str(tmp_path / "missing.bin"), 1, 3)
