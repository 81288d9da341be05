"""The C-ABI library loads and exports every function include/*.h declares
(no compute calls: these run without a GPU)."""
import re
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(ld_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_the_pipeline():
    names = declared_functions()
    for n in ["ld_problem_from_file", "ld_problem_check_launch", "ld_problem_solve",
              "ld_solve_reduced", "ld_problem_report", "ld_plan_create", "ld_cli_main"]:
        assert n in names


def test_library_exports_every_declared_symbol(ld):
    lib = ld.lib()
    exported = subprocess.run(["nm", "-D", "--defined-only", str(ld.LIB_PATH)], capture_output=True,
                              text=True, check=True).stdout
    for name in declared_functions():
        assert getattr(lib, name) is not None
        assert re.search(rf"\bT {name}$", exported, flags=re.M), name


def test_binding_covers_every_declared_symbol(ld):
    bound = {n for n, _, _ in ld.SIGNATURES}
    assert declared_functions() <= bound


def test_version_and_error_strings(ld):
    assert b"sm_100a" in ld.lib().ld_version()
    assert ld.lib().ld_last_error() is not None
