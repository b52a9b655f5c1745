"""The drop-in CLI (hero_b200/bin/hero_b200): flag handling without a GPU."""
import os
import subprocess

import pytest

from hero_b200 import build


@pytest.fixture(scope="module")
def cli():
    build.build_library()
    path = build.build_cli()
    assert path and os.path.exists(path)
    return path


def run(cli, *args):
    return subprocess.run([cli, *args], capture_output=True, text=True)


def test_help(cli):
    r = run(cli, "--help")
    assert r.returncode == 1 and "Usage" in r.stdout


def test_requires_inputs(cli):
    r = run(cli, "-c")
    assert r.returncode == 1 and "missed -subject or -query" in r.stderr


def test_alignment_output_mode_without_c(cli, tmp_path):
    # no -c: the .aln mode; the flags parse and the run stops at the missing input
    r = run(cli, "-q", str(tmp_path / "nope.fq"), "-s", str(tmp_path / "nope.fq"))
    assert r.returncode == 1 and "Unable to open file" in r.stderr


@pytest.mark.parametrize("flag", ["-v", "--covfilter", "--suffix"])
def test_refuses_modes_outside_the_path(cli, flag):
    r = run(cli, "-q", "a.fq", "-s", "a.fq", "-c", flag)
    assert r.returncode == 1 and "not part of the path" in r.stderr


def test_missing_file(cli, tmp_path):
    r = run(cli, "-q", str(tmp_path / "nope.fq"), "-s", str(tmp_path / "nope.fq"), "-c")
    assert r.returncode == 1 and "Unable to open file" in r.stderr
