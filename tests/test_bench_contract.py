"""CPU checks of bench.py's contract: every name the functions of bench.py,
the build entry and the Python packages read is defined (a static scan of
the modules' scopes), and the reference arm --
the reference's own CPU code on the default workload -- runs and prints one
JSON line with the fields the contract asks for."""
import builtins
import json
import os
import subprocess
import symtable
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def undefined_globals(path):
    """(scope, name) of every implicit global a function reads that the
    module neither defines nor imports and that is not a builtin."""
    src = open(path).read()
    top = symtable.symtable(src, path, "exec")
    defined = {s.get_name() for s in top.get_symbols() if s.is_assigned() or s.is_imported() or s.is_namespace()}
    out = []

    def walk(t):
        for s in t.get_symbols():
            n = s.get_name()
            if s.is_global() and not s.is_declared_global() and s.is_referenced() and n not in defined \
                    and not hasattr(builtins, n) and n != "__file__":
                out.append((t.get_name(), n))
        for c in t.get_children():
            walk(c)

    walk(top)
    return out


@pytest.mark.parametrize("name", ["bench.py", "__graft_entry__.py"] + sorted(
    os.path.join(d, f) for d in ("timbir_b200", "oracle") for f in os.listdir(os.path.join(ROOT, d))
    if f.endswith(".py")))
def test_entry_scripts_read_no_undefined_name(name):
    assert undefined_globals(os.path.join(ROOT, name)) == []


def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(s) for s in r.stdout.splitlines() if s.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and "unavailable" not in d
    assert d["metric"] == "ICD voxel-updates/s" and d["unit"] == "voxel-updates/s" and d["value"] > 0
    assert d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["e2e"]["d2h_bytes_per_step"] == 0
