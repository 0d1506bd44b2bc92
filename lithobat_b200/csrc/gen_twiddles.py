"""Write twiddles.cuh: the 64th roots of unity as FP32 literals, and the
ratio of their smaller to their larger component (for factored twiddles).

cos/sin(2*pi*k/64) are evaluated in FP64 by the host's libm and printed with
17 significant digits, so the compiler's decimal-to-float conversion gives
the correctly rounded FP32 value. Run by the build step.
"""
import math
import sys
from pathlib import Path


def main(out: Path) -> None:
    lines = [
        "// Generated by gen_twiddles.py. exp(2*pi*i*k/64) for k = 0..63.",
        "#pragma once",
        "namespace litho {",
        "__device__ __forceinline__ float tw64_re(int k) {",
        "  switch (k & 63) {",
    ]
    for k in range(64):
        lines.append(f"    case {k}: return {math.cos(2 * math.pi * k / 64):.17e}f;")
    lines += ["  }", "  return 0.f;", "}", "__device__ __forceinline__ float tw64_im(int k) {",
              "  switch (k & 63) {"]
    for k in range(64):
        lines.append(f"    case {k}: return {math.sin(2 * math.pi * k / 64):.17e}f;")
    lines += ["  }", "  return 0.f;", "}",
              "// sin/cos where |cos| >= |sin| (tw64_cos_major), else cos/sin: |ratio| <= 1.",
              "__host__ __device__ constexpr bool tw64_cos_major(int k) {",
              "  return (k & 31) <= 8 || (k & 31) >= 24;",
              "}",
              "__device__ __forceinline__ float tw64_ratio(int k) {",
              "  switch (k & 63) {"]
    for k in range(64):
        c, s = math.cos(2 * math.pi * k / 64), math.sin(2 * math.pi * k / 64)
        cos_major = (k & 31) <= 8 or (k & 31) >= 24
        assert cos_major == (abs(c) >= abs(s) - 1e-15)
        lines.append(f"    case {k}: return {(s / c if cos_major else c / s):.17e}f;")
    lines += ["  }", "  return 0.f;", "}", "}  // namespace litho", ""]
    out.write_text("\n".join(lines))


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).with_name("twiddles.cuh"))
