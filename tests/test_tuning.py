"""The tuning table (dgpu_tuning_*): per read-length class launch shapes,
their text file, and input checks. CPU only: the table is host state, and
results never depend on it (the GPU parity tests run under whatever table is
in force)."""
import pytest

import dada2_b200 as D


@pytest.fixture
def saved_table(tmp_path):
    keep = tmp_path / "keep.txt"
    D.tuning_save(str(keep))
    yield tmp_path
    D.tuning_load(str(keep))


def test_classes_follow_read_length(saved_table):
    assert [D.length_class(n) for n in (1, 150, 200, 201, 250, 600, 601, 1450)] == [0, 0, 0, 1, 1, 1, 2, 2]
    s150 = {**D.tuning_get(150), "launch_slots": 3, "align_ctas_per_sm": 2}
    D.tuning_set(0, s150)
    assert D.tuning_get(150) == s150
    assert D.tuning_get(200) == s150
    assert D.tuning_get(250) != s150 or D.tuning_get(250)["launch_slots"] == 3


def test_save_and_load_round_trip(saved_table):
    path = saved_table / "t.txt"
    a = {"launch_slots": 8, "samples_per_launch": 2, "dedicated_slots": 0, "align_ctas_per_sm": 3,
         "screen_chunk_max": 16, "screen_blocks_per_sm": 2, "pivot_min_items": 4096,
         "programmatic_launch": 0}
    b = {**a, "launch_slots": 4, "samples_per_launch": 16, "dedicated_slots": 2}
    D.tuning_set(1, a)
    D.tuning_set(2, b)
    D.tuning_save(str(path))
    text = path.read_text()
    assert "class 1 launch_slots 8 samples_per_launch 2" in text
    D.tuning_reset()
    assert D.tuning_get(250) != a
    D.tuning_load(str(path))
    assert D.tuning_get(250) == a and D.tuning_get(1450) == b


def test_partial_lines_keep_other_keys(saved_table):
    path = saved_table / "p.txt"
    D.tuning_reset()
    before = D.tuning_get(150)
    path.write_text("# only one knob of class 0\nclass 0 launch_slots 2\n")
    D.tuning_load(str(path))
    assert D.tuning_get(150) == {**before, "launch_slots": 2}


@pytest.mark.parametrize("text,why", [
    ("class 3 launch_slots 2\n", "class must be"),
    ("class 0 launch_slots 9\n", "out of range"),
    ("class 0 screen_chunk_max 24\n", "out of range"),
    ("class 0 align_ctas_per_sm 0\n", "out of range"),
    ("class 0 pivot_min_items -1\n", "out of range"),
    ("class 0 programmatic_launch 2\n", "out of range"),
    ("class 0 warp_size 16\n", "unknown key"),
    ("launch_slots 2\n", "expected"),
])
def test_malformed_files_are_rejected_and_change_nothing(saved_table, text, why):
    path = saved_table / "bad.txt"
    path.write_text(text)
    before = [D.tuning_get(n) for n in (150, 250, 1450)]
    with pytest.raises(D.InvalidInput, match=why):
        D.tuning_load(str(path))
    assert [D.tuning_get(n) for n in (150, 250, 1450)] == before


def test_set_rejects_out_of_range_values(saved_table):
    bad = {**D.tuning_get(150), "samples_per_launch": 0}
    with pytest.raises(D.InvalidInput):
        D.tuning_set(0, bad)
    with pytest.raises(D.InvalidInput):
        D.tuning_set(3, D.tuning_get(150))
