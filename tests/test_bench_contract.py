"""bench.py's structure (CPU): one definition per top-level name (a second
definition would silently replace the first) and a command line that parses
the driver's flags and the studies."""
import ast
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_no_top_level_name_defined_twice():
    tree = ast.parse(open(os.path.join(REPO, "bench.py")).read())
    names = [n.name for n in tree.body if isinstance(n, (ast.FunctionDef, ast.ClassDef))]
    dup = sorted({n for n in names if names.count(n) > 1})
    assert not dup, dup


def test_command_line_parses():
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--help"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    for flag in ("--gpus", "--steps", "--warmup", "--impl", "--study", "--no-autotune"):
        assert flag in r.stdout
    assert "winc_sweep" in r.stdout and "baselines" in r.stdout
