"""The ctypes mirrors of the C-ABI structures have the header's layout: a small C program built
against include/dirac_gpu.h with the host compiler prints every structure's size and each
field's offset, by the field names the Python binding uses, and they must equal ctypes'.  A
field renamed, reordered, retyped or appended on one side only fails here.  No GPU use."""
import ctypes
import keyword
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "dirac-research_b200"))


def _mirrors():
    from dirac_b200._lib import BlockParams
    from dirac_b200.batch import BatchMotion, BatchPicture
    from dirac_b200.decoder import DecodeInput, DecoderParams
    from dirac_b200.encoder import EncoderParams, PictureInfo

    return {"dgpu_block_params": BlockParams, "dgpu_encoder_params": EncoderParams,
            "dgpu_picture_info": PictureInfo, "dgpu_batch_picture": BatchPicture,
            "dgpu_batch_motion": BatchMotion, "dgpu_decoder_params": DecoderParams,
            "dgpu_decode_input": DecodeInput}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs the host C compiler")
def test_ctypes_structures_match_the_header(tmp_path):
    mirrors = _mirrors()
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "dirac_gpu.h"', "int main(void) {"]
    want = []
    for cname, cls in mirrors.items():
        lines.append(f'    printf("%zu\\n", sizeof({cname}));')
        want.append(ctypes.sizeof(cls))
        for field in cls._fields_:
            name = field[0]
            # a C field named like a Python keyword is mirrored with a trailing underscore
            c_field = name[:-1] if name.endswith("_") and keyword.iskeyword(name[:-1]) else name
            lines.append(f'    printf("%zu\\n", offsetof({cname}, {c_field}));')
            want.append(getattr(cls, name).offset)
    lines += ["    return 0;", "}"]
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "abi"
    cc = subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == want
