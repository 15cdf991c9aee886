"""Build recipe: the reference's own hot-path compute shaders as C++.

The non-uniform collocated shader (FvmCollNonUniform.compute) is translated
beside the uniform one.

Reads the shader sources where they lie in the reference checkout and writes
C++ translations into oracle/_ref/ (never committed): the HLSL subset these
kernels use maps onto oracle/hlsl_shim.h after a few textual rewrites
(constants include inlined, kernel pragmas, thread-count attributes and
system-value semantics dropped, `.xyz` swizzles made calls, float literals
given the single-precision suffix).  oracle/ref_driver.cpp includes the
results and dispatches the kernels in the order of FvmSolverGpu.Step.

    python oracle/ref_kernels.py [reference_root]
"""
from __future__ import annotations

import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHADER_DIR = "Assets/Resources/Shaders"
SHADERS = {
    "fvm": "SimShaders/FvmColl.compute",
    "fvmnu": "SimShaders/FvmCollNonUniform.compute",
    "piso": "SimShaders/PisoColl.compute",
    "les": "LESShaders/LES.compute",
    "wall": "WallFuncShaders/WallFunc.compute",
    "utils": "SimShaders/Utils.compute",
    "init": "InitShaders/InitShaderColl.compute",
}
CONSTANTS = "Includes/Constants.hlsl"

_FLOAT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")


def translate(text: str, constants: str) -> str:
    text = re.sub(r'#include\s+"[^"]*Constants\.hlsl"', lambda m: constants, text)
    text = re.sub(r"\bstatic const\b", "static constexpr", text)
    text = re.sub(r"^\s*#pragma\s+kernel.*$", "", text, flags=re.M)
    text = re.sub(r"\[numthreads\([^)]*\)\]", "", text)
    text = re.sub(r":\s*SV_\w+", "", text)
    text = re.sub(r"\.xyz\b(?!\s*\()", ".xyz()", text)
    text = _FLOAT.sub(lambda m: m.group(1) + "f", text)
    return text


def generate(ref_root: str) -> list[str]:
    os.makedirs(OUT, exist_ok=True)
    base = os.path.join(ref_root, SHADER_DIR)
    with open(os.path.join(base, CONSTANTS)) as f:
        # the include guard is dropped: each shader gets its own copy
        constants = re.sub(r"^\s*#(ifndef|define|endif)\b.*$", "", f.read(), flags=re.M)
        constants = translate(constants, "")
    written = []
    for name, rel in SHADERS.items():
        with open(os.path.join(base, rel)) as f:
            src = f.read()
        path = os.path.join(OUT, f"{name}.inc")
        with open(path, "w") as f:
            f.write(f"// generated by oracle/ref_kernels.py from {SHADER_DIR}/{rel}\n")
            f.write(translate(src, constants))
        written.append(path)
    return written


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: ref_kernels.py <reference checkout root>")
    root = sys.argv[1]
    for p in generate(root):
        print(p)
