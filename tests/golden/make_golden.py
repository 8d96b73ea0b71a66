"""Regenerates the golden files of tests/golden from CODAG's own Python compressors.

Runs only where the CODAG tree is available: give it with --ref or $CODAG_REFERENCE_DIR.
deflate_compressor.py imports `zstandard` at module level without using it on this path,
and writes to a hard-coded directory; the script stubs the first and redirects the second
into this folder, then calls CODAG's zlib_chunk_compress (deflate_compressor.py:44-125)
on a seeded text sample; likewise rapids_compressor.py's zlib_chunk_compress
(rapids_compressor.py:222-275, the layout of CODAG's cuDF comparison, 64 KiB chunks at zlib
level 9), which writes output/comp3.bin under the working directory, run in a temporary
directory.  The tests compare our layout writers against these files.

    CODAG_REFERENCE_DIR=<CODAG tree> python tests/golden/make_golden.py
"""
import builtins
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def main() -> None:
    ref = sys.argv[sys.argv.index("--ref") + 1] if "--ref" in sys.argv else os.environ.get("CODAG_REFERENCE_DIR")
    if not ref:
        sys.exit("give the CODAG source tree with --ref or CODAG_REFERENCE_DIR")
    REF = Path(ref)
    sys.path.insert(0, str(REPO))
    from codag_b200 import native

    src = native.gen_text(140_000, 424242)
    (HERE / "deflate_src.bin").write_bytes(src.tobytes())

    sys.modules.setdefault("zstandard", types.ModuleType("zstandard"))
    sys.path.insert(0, str(REF))
    import deflate_compressor as dc  # CODAG's compressor

    prefix = "/home/jpark346/compressor/output/"

    def redirected_open(path, *args, **kwargs):
        if isinstance(path, str) and path.startswith(prefix):
            path = str(HERE / path[len(prefix):])
        return builtins.open(path, *args, **kwargs)

    dc.open = redirected_open
    dc.print = lambda *a, **k: None
    dc.zlib_chunk_compress(src.tobytes(), "deflate_ref")
    for name in ("deflate_ref_comp.bin", "deflate_ref_blk_offset.bin", "deflate_ref_col_len.bin"):
        print(name, (HERE / name).stat().st_size)

    import tempfile
    import rapids_compressor as rc  # CODAG's cuDF-comparison compressor
    rc.print = lambda *a, **k: None
    cudf_src = native.gen_text(200_000, 434343)
    (HERE / "cudf_src.bin").write_bytes(cudf_src.tobytes())
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as td:
        os.chdir(td)
        try:
            os.mkdir("output")
            rc.zlib_chunk_compress(cudf_src.tobytes())
            (HERE / "cudf_ref_comp.bin").write_bytes(Path(td, "output", "comp3.bin").read_bytes())
        finally:
            os.chdir(cwd)
    print("cudf_ref_comp.bin", (HERE / "cudf_ref_comp.bin").stat().st_size)


if __name__ == "__main__":
    main()
