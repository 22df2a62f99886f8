"""Writes isaacb_blue_noise.h: the 8^3 and 16^3 blue-noise dither masks that the
reference vendors in lib/isaac/isaac_dither_kernel.hpp (dither modes 3 and >= 4;
generated there with the MomentsInGraphics BlueNoise tool).  The masks decide the
output bytes of those modes, so they are kept identical.

    python isaac_b200/csrc/gen_blue_noise.py <reference tree>/lib/isaac/isaac_dither_kernel.hpp
"""

import re
import sys
from pathlib import Path


def tables(text: str):
    found = re.findall(r"static const isaac_ushort ditherMask\[(\d+)\]\s*=\s*\{([^}]*)\}", text)
    out = {}
    for n, body in found:
        vals = [int(v) for v in re.findall(r"\d+", body)]
        assert len(vals) == int(n), (n, len(vals))
        out[int(n)] = vals
    assert set(out) == {512, 4096}, sorted(out)
    return out


def main(src: str):
    t = tables(Path(src).read_text())
    lines = [
        "// Generated by gen_blue_noise.py from the reference's dither kernel",
        "// (lib/isaac/isaac_dither_kernel.hpp, dither modes 3 and >= 4): 8^3 and 16^3",
        "// blue-noise masks, x fastest, then y, then z.  Do not edit.",
        "#pragma once",
        "",
        "#include <cstdint>",
        "",
    ]
    for n, name in ((512, "8"), (4096, "16")):
        lines.append(f"#define ISAACB_BLUE_NOISE{name}_VALUES \\")
        vals = t[n]
        for i in range(0, n, 16):
            tail = ", \\" if i + 16 < n else ""
            lines.append("    " + ", ".join(str(v) for v in vals[i : i + 16]) + tail)
        lines.append("")
        lines.append(f"static const uint16_t kBlueNoise{name}[{n}] = {{ISAACB_BLUE_NOISE{name}_VALUES}};")
        lines.append("")
    out = Path(__file__).resolve().parent / "isaacb_blue_noise.h"
    out.write_text("\n".join(lines))
    print(out)


if __name__ == "__main__":
    main(sys.argv[1])
