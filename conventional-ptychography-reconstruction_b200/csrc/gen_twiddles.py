"""Generate twiddle4096.cuh: exp(-2 pi i k / 4096), k = 0..4095, as float2.

    python conventional-ptychography-reconstruction_b200/csrc/gen_twiddles.py

Each entry is cos / sin of 2 pi k / 4096 evaluated in double precision (Python's
math library) and rounded once to float32, so the table is the correctly
rounded one the power-of-two Fourier resampling kernels (resample.cu) index
with stride 4096 / L for every line length L <= 4096.  The table is a
statically initialised __device__ array: no run-time set-up, and a new CUDA
context (after a device reset) loads it again with the module.
"""
import math
import os
import struct

N = 4096
HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "twiddle4096.cuh")


def f32(x: float) -> float:
    return struct.unpack("<f", struct.pack("<f", x))[0]


def lit(x: float) -> str:
    # shortest decimal that reads back as the same float32 (9 significant digits always do)
    v = f32(x)
    if v == 0.0:
        return "0.0f"
    t = f"{v:.9g}"
    if "." not in t and "e" not in t:
        t += ".0"  # "1f" is not a floating literal
    return t + "f"


def main() -> None:
    lines = []
    for k in range(N):
        # exp(-2 pi i k / N): use the exact symmetries for the axis points
        if k == 0:
            c, s = 1.0, 0.0
        elif k == N // 4:
            c, s = 0.0, -1.0
        elif k == N // 2:
            c, s = -1.0, 0.0
        elif k == 3 * N // 4:
            c, s = 0.0, 1.0
        else:
            a = 2.0 * math.pi * k / N
            c, s = math.cos(a), -math.sin(a)
        lines.append(f"    {{{lit(c)}, {lit(s)}}},")
    body = "\n".join(lines)
    text = (
        "// twiddle4096.cuh -- generated by gen_twiddles.py; do not edit.\n"
        "// kTw4096[k] = exp(-2 pi i k / 4096), cos and sin in double precision\n"
        "// rounded once to float32.\n"
        "#pragma once\n"
        "#include <cuda_runtime.h>\n\n"
        "namespace pty {\n\n"
        f"__device__ const float2 kTw4096[{N}] = {{\n{body}\n}};\n\n"
        "}  // namespace pty\n"
    )
    with open(OUT, "w") as f:
        f.write(text)


if __name__ == "__main__":
    main()
