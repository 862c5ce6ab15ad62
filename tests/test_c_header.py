"""include/turing_sht.h from a plain C caller: the header compiles as C99
with -pedantic -Werror, a program using it links against libturing_sht.so,
and its GPU-free calls (layout algebra, seeding, error paths) return what the
reference's rules say.  No GPU needed (ts_ctx_create's status is reported,
whichever it is)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "turing_sphere_b200")


def test_header_compiles_links_and_runs_as_plain_c(tmp_path):
    exe = tmp_path / "header_check"
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_abi", "header_check.c"),
                    "-o", str(exe), "-L", LIBDIR, "-lturing_sht", "-lm",
                    f"-Wl,-rpath,{LIBDIR}"], check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")
