"""CPU checks of the command-line front end: it builds, and argument errors
are reported before any device work (no GPU needed)."""
import os
import subprocess

import pytest

from conftest import ROOT

CLI = os.path.join(ROOT, "isp_mw_b200", "lib", "isp_mw")


@pytest.fixture(scope="module")
def cli(bm3d_lib):
    assert os.access(CLI, os.X_OK)
    return CLI


def run(cli, *args):
    return subprocess.run([cli] + list(args), capture_output=True, text=True, timeout=60)


def test_usage_and_unknown_filter(cli):
    r = run(cli)
    assert r.returncode == 0 and "Not enough arguments" in r.stdout
    r = run(cli, "--nlmeans", "x.png")
    assert r.returncode == 1 and "not part of this build" in r.stderr


@pytest.mark.parametrize("args,msg", [
    (["x.raw"], "--width and --height"),
    (["-W", "8", "-H", "8"], "no input"),
    (["-W", "8", "-H", "8", "--type", "cmyk", "x.raw"], "unknown --type"),
    (["-W", "8", "-H", "8", "--depth", "20", "x.raw"], "--depth"),
    (["-W", "eight", "-H", "8", "x.raw"], "bad integer"),
    (["-P", "ultra", "x.raw"], "unrecognized profile"),
    (["-W", "8", "-H", "8", "--bogus", "1", "x.raw"], "unknown option"),
    (["-W", "8", "-H", "8", "/nonexistent/x.raw"], "cannot open"),
])
def test_argument_errors(cli, args, msg):
    r = run(cli, "--bm3d", *args)
    assert r.returncode == 2 and msg in r.stderr, (r.returncode, r.stderr)
