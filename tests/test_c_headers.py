"""The public headers are plain C: every include/*.h compiles as C99 and as
C++11 with -pedantic, and a C program links against libdygrass.so and gets
the documented argument errors from calls that need no GPU."""
import os
import shutil
import subprocess

import pytest

import dygrass_b200 as dyg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "dyg.h"
#include "dyg_io.h"
#include "dyg_serve.h"

int main(void) {
    dyg_walk_params p;
    dyg_walk_params_default(&p);
    if (p.walkers != 512 || p.max_steps != 100) return 1;
    if (strstr(dyg_version(), "sm_100a") == NULL) return 2;
    dyg_server *s = NULL;
    uint32_t off[2] = {0, 4};
    if (dyg_server_create(NULL, NULL, 1, off, &p, &p, NULL, &s) != DYG_EINVAL || s != NULL) return 3;
    if (strlen(dyg_last_error_string()) == 0) return 4;
    if (dyg_server_submit(NULL, 0, 0, DYG_STREAM_INSERT, NULL, NULL, NULL, 0) != DYG_EINVAL) return 5;
    if (dyg_server_pending(NULL) != 0 || dyg_server_steps(NULL) != 0) return 6;
    if (dyg_server_destroy(NULL) != DYG_OK) return 7;
    if (dyg_reference_batch_size(95) != 10) return 8;
    puts("ok");
    return 0;
}
"""


def _cc(name):
    path = shutil.which(name)
    if not path:
        pytest.skip(f"{name} not found")
    return path


@pytest.mark.parametrize("lang", ["c99", "c++11"])
def test_headers_compile_pedantic(tmp_path, lang):
    src = tmp_path / "all.c"
    src.write_text("".join(f'#include "{h}"\n' for h in sorted(os.listdir(INC)) if h.endswith(".h"))
                   + "int main(void) { return 0; }\n")
    if lang == "c99":
        cmd = [_cc("gcc"), "-std=c99"]
    else:
        cmd = [_cc("g++"), "-std=c++11", "-x", "c++"]
    cmd += ["-Wall", "-Wextra", "-pedantic", "-Werror", "-I", INC, "-c", str(src), "-o",
            str(tmp_path / "all.o")]
    cp = subprocess.run(cmd, capture_output=True, text=True)
    assert cp.returncode == 0, cp.stderr


def test_c_program_links_and_checks_arguments(tmp_path):
    src = tmp_path / "prog.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "prog"
    libdir = os.path.dirname(dyg.LIB_PATH)
    cp = subprocess.run([_cc("gcc"), "-std=c99", "-I", INC, str(src), "-o", str(exe), "-L", libdir,
                         "-ldygrass", f"-Wl,-rpath,{libdir}"], capture_output=True, text=True)
    assert cp.returncode == 0, cp.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and run.stdout.strip() == "ok", (run.returncode, run.stdout, run.stderr)
