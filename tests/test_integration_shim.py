"""The HYPRE-side hook code of INTEGRATION.md compiles (CPU test): every
```c block of the document, in order, is compiled as one translation unit
against include/amgt_b200.h and HYPRE-shaped declarations
(tests/hypre_shim/hypre_subset.h, after AmgT_HYPRE/src/seq_mv/seq_mv.h),
with warnings as errors, so that the shim text a maintainer copies cannot
drift from the library's signatures."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_integration_c_blocks_compile(tmp_path):
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```c\n(.*?)```", text, flags=re.S)
    assert len(blocks) >= 6
    body = ["#include \"hypre_subset.h\"", "HYPRE_Int hypre_error_flag;"]
    for b in blocks:
        if b.strip().startswith("#include \"amgt_b200.h\""):
            continue  # section 1: the typedef the subset header already makes
        body.append(b)
    # reference every static function so that -Wunused-function stays quiet
    names = re.findall(r"^static\s+[\w\s\*]+?\b(\w+)\s*\(", "\n".join(body), flags=re.M)
    body.append("void *amgt_shim_uses[] = {" + ", ".join(f"(void *){n}" for n in names) + "};")
    src = tmp_path / "shim.c"
    src.write_text("\n".join(body))
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-Wno-unused-parameter", "-c",
                        "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "tests", "hypre_shim"),
                        str(src), "-o", str(tmp_path / "shim.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
