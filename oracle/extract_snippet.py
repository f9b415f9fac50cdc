"""TEST INFRASTRUCTURE: pull an application's GLSL fetch snippet out of its
C++ source (oracle/Makefile runs this on the HPMC tree).

The reference's demo applications pass their custom-fetch GLSL to
HPMCsetFieldCustom as a C++ std::string initialised by concatenated string
literals (e.g. apps/cayley/cayley.cpp:75-94).  This reads that initialiser
from the application's source as text and writes the GLSL it denotes, so the
custom-fetch tests run the reference's own snippet through the reference's
own shader generator; nothing is copied into the repository (the output goes
to oracle/_ref/, which is git-ignored).

    python extract_snippet.py <source.cpp> <variable name> <output.glsl>
"""
from __future__ import annotations

import re
import sys


def snippet(cpp_text: str, name: str) -> str:
    m = re.search(r"std::string\s+" + re.escape(name) + r"\s*=(.*?);\s*\n", cpp_text, flags=re.S)
    if not m:
        raise ValueError(f"no std::string {name} initialiser")
    body = re.sub(r"//[^\n]*", "", m.group(1))  # comments between the literals
    parts = re.findall(r'"((?:[^"\\]|\\.)*)"', body)
    return "".join(bytes(p, "utf-8").decode("unicode_escape") for p in parts)


def main(argv: list[str]) -> int:
    src, name, out = argv[1:4]
    with open(src) as f:
        text = snippet(f.read(), name)
    with open(out, "w") as f:
        f.write(text)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
