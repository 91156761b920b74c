"""Restart files in the reference's format (CPU): the TorchScript tensor
archive of one block, the part names, the bundle of several blocks and its
header, and reading a block back from a bundle or a single part."""
import os

import pytest

from snapy_linfel_b200 import restart

torch = pytest.importorskip("torch")


def _vars(seed, scalars=True):
    g = torch.Generator().manual_seed(seed)
    v = {"hydro_u": torch.randn(5, 4, 6, 8, generator=g, dtype=torch.float64),
         "hydro_w": torch.randn(5, 4, 6, 8, generator=g, dtype=torch.float64)}
    if scalars:
        v["scalar_s"] = torch.rand(2, 4, 6, 8, generator=g, dtype=torch.float64)
        v["scalar_r"] = torch.rand(2, 4, 6, 8, generator=g, dtype=torch.float64)
    return v


def test_archive_round_trip(tmp_path):
    p = str(tmp_path / "a.part")
    v = _vars(1)
    restart.save_tensors(v, p)
    back = restart.load_tensors(p)
    assert set(back) == set(v)
    for k in v:
        assert back[k].dtype == v[k].dtype and torch.equal(back[k], v[k])


def test_part_names():
    assert restart.part_name("straka", 3, 7) == "straka.block3.00007.part"
    assert restart.part_name("straka", 0, 7, final=True) == "straka.block0.final.part"
    assert restart.parse_part_name("a.b.block12.00003.part") == ("a.b", 12, "00003")
    with pytest.raises(ValueError):
        restart.parse_part_name("straka.00003.restart")


def test_part_contents(tmp_path):
    v = _vars(2)
    p = restart.write_part(v, str(tmp_path), "run", rank=1, file_number=4, current_time=12.5,
                           cycle=40, output_file_numbers=[4, 9], output_next_times=[15.0, 20.0])
    assert os.path.basename(p) == "run.block1.00004.part"
    back = restart.load_tensors(p)
    # scalar_r is derived from scalar_s and hydro_u, so it is not stored
    assert set(back) == {"hydro_u", "hydro_w", "scalar_s", "last_time", "last_cycle",
                         "file_number", "next_time"}
    assert float(back["last_time"][0]) == 12.5 and int(back["last_cycle"][0]) == 40
    assert back["last_cycle"].dtype == torch.int64 and back["last_time"].dtype == torch.float64
    assert back["file_number"].tolist() == [4, 9] and back["next_time"].tolist() == [15.0, 20.0]
    assert torch.equal(back["hydro_u"], v["hydro_u"])


def test_bundle_and_single(tmp_path):
    d = str(tmp_path)
    vs = [_vars(10 + r, scalars=False) for r in range(3)]
    for r, v in enumerate(vs):
        restart.write_part(v, d, "run", rank=r, file_number=2, current_time=1.0 + r, cycle=5)
    out = restart.combine(d, "run", 2)
    assert os.path.basename(out) == "run.00002.restart"
    assert not any(f.endswith(".part") for f in os.listdir(d))  # parts removed
    with open(out, "rb") as f:
        head = f.read(200).split(b"\n")
    assert head[0] == b"SNAPY_RESTART_BUNDLE_V1" and head[1] == b"3"
    names = [h.split(b"\t")[0] for h in head[2:5]]
    assert names == [b"run.block0.00002.part", b"run.block1.00002.part",
                     b"run.block2.00002.part"]
    assert restart.is_bundle(out)
    for r in (2, 0, 1):
        back = restart.load_restart(out, r)
        assert torch.equal(back["hydro_u"], vs[r]["hydro_u"])
        assert float(back["last_time"][0]) == 1.0 + r
    with pytest.raises(KeyError):
        restart.load_restart(out, 5)
    # one block: the part itself becomes the restart file
    restart.write_part(vs[0], d, "solo", rank=0, file_number=0, current_time=0.0, cycle=0,
                       final=True)
    single = restart.combine(d, "solo", 0, final=True)
    assert os.path.basename(single) == "solo.final.restart" and not restart.is_bundle(single)
    assert torch.equal(restart.load_restart(single, 0)["hydro_w"], vs[0]["hydro_w"])


def _ref_fixture():
    import sys

    here = os.path.join(os.path.dirname(__file__), "golden")
    sys.path.insert(0, here)
    try:
        import make_restart_fixture as m
    finally:
        sys.path.remove(here)
    return os.path.join(here, "ref_restart.block0.00003.part"), m.fixture_tensors()


def test_reads_a_part_written_by_the_reference(tmp_path):
    """a restart part written by the reference's own save_tensors
    (python/write_init.py:12-22) is read back exactly, as a single part and
    from a bundle, and restores like one written here"""
    path, want = _ref_fixture()
    back = restart.load_restart(path, 0)
    assert set(back) == set(want)
    for k, v in want.items():
        assert back[k].dtype == v.dtype and torch.equal(back[k], v), k
    # bundled with two parts written here, it is found by its block rank
    d = str(tmp_path)
    import shutil

    shutil.copy(path, os.path.join(d, "ref.block0.00003.part"))
    for r in (1, 2):
        restart.write_part(_vars(20 + r), d, "ref", rank=r, file_number=3, current_time=1.0,
                           cycle=2)
    out = restart.combine(d, "ref", 3)
    got = restart.load_restart(out, 0)
    assert torch.equal(got["hydro_u"], want["hydro_u"]) and int(got["last_cycle"][0]) == 77
    # the same variables written here give the same buffers
    mine = str(tmp_path / "mine.part")
    restart.save_tensors(want, mine)
    again = restart.load_tensors(mine)
    assert all(torch.equal(again[k], want[k]) for k in want)
