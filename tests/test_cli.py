"""The ./method driver: cache files, command line and output record."""
import filecmp
import os
import shutil
import subprocess

import pytest

import lpa_b200 as L
from conftest import GOLDEN

EXTS = [".graph", ".offset", ".vertices.bin", ".row", ".clm"]


def _run(tmp_path, args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([str(L.METHOD_PATH), *args], cwd=tmp_path, capture_output=True, text=True, env=e,
                          timeout=600)


def test_cli_writes_reference_cache_files(tmp_path):
    """Without cache files the driver ingests the edge list and writes the same
    .graph/.offset/.vertices.bin/.row/.clm as the reference (File::write_binary)."""
    src = GOLDEN / "road_b" / "g.txt"
    shutil.copy(src, tmp_path / "g.txt")
    r = _run(tmp_path, ["g.txt", "1", "1", "0", "out.txt"])
    for ext in EXTS:
        assert filecmp.cmp(str(src) + ext, str(tmp_path / "g.txt") + ext, shallow=False), ext
    assert "Input graph check:" in r.stdout


@pytest.mark.gpu
def test_cli_runs_and_appends_record(tmp_path):
    src = GOLDEN / "road_a" / "g.txt"
    shutil.copy(src, tmp_path / "g.txt")
    r = _run(tmp_path, ["g.txt", "1", "0", "0", "out.txt"])
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ": " in ln and "(ms), updated" in ln]
    assert len(lines) == 20 and lines[0].startswith("1: ")
    assert "f1: " in r.stdout and ",f2: " in r.stdout
    rec = (tmp_path / "out.txt").read_text().splitlines()
    assert rec[0] == "nova file: g.txt"
    assert rec[1].startswith(" running time: ") and rec[1].endswith("thre: 0")
    assert rec[2] == "~~~~~"
    # the two-pass driver name
    os.symlink(L.METHOD_PATH, tmp_path / "cglp")
    r = subprocess.run([str(tmp_path / "cglp"), "g.txt", "1", "0", "0", "out.txt"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "out.txt").read_text().splitlines()[3] == "cglp file: g.txt"
