"""TEST INFRASTRUCTURE ONLY: rewrite the reference's HLSL sources into C++ that compiles against the
GPRT stand-in (oracle/hlsl/gprt.h), so the reference's own device programs run on the CPU.

    python oracle/hlsl/hlsl2cpp.py <reference tree> <output dir>

Reads sharedCode.h, rng.h and the four deviceCode*.hlsl modules where they lie in the reference
tree and writes the rewritten text to <output dir> (oracle/_ref/hlsl, git-ignored). The rewrite is
purely syntactic -- HLSL constructs that C++ spells differently -- and changes no computation:

  - `[raypayload]` and `[[vk::push_constant]]` annotations are dropped;
  - `class` becomes `struct` (HLSL class members are public);
  - parameter qualifiers: `in T x` -> `const T &x`, `out T x` / `inout T x` -> `T &x`;
  - unsuffixed floating literals get an `f` suffix: HLSL gives an unsuffixed literal the type of
    the float expression it meets (a `literal float`), where C++ would promote the whole
    expression to double;
  - `1.#INF` (HLSL's infinity literal) becomes INFINITY.
"""
import os
import re
import sys

FILES = ["sharedCode.h", "rng.h", "deviceCodeRBF.hlsl", "deviceCodeSplat.hlsl", "deviceCodeCommon.hlsl",
         "deviceCodeBounds.hlsl"]

FLOAT_LIT = re.compile(r"(?<![\w.#])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.#])")
PARAM = re.compile(r"([(,]\s*)(inout|out|in)\s+([A-Za-z_]\w*)\s+([A-Za-z_]\w*)")


def rewrite(text: str) -> str:
    text = text.replace("[raypayload]", "")
    text = text.replace("[[vk::push_constant]]", "")
    text = text.replace("1.#INF", "INFINITY")
    text = re.sub(r"\bclass\b", "struct", text)

    def param(m):
        q, t, n = m.group(2), m.group(3), m.group(4)
        return f"{m.group(1)}{'const ' if q == 'in' else ''}{t} &{n}"

    text = PARAM.sub(param, text)
    out = []
    for line in text.split("\n"):
        # leave preprocessor lines and // comments as they are
        code, sep, comment = line.partition("//")
        if code.lstrip().startswith("#"):
            out.append(line)
            continue
        code = FLOAT_LIT.sub(lambda m: m.group(1) + "f", code)
        out.append(code + sep + comment)
    return "\n".join(out)


def main():
    ref, dst = sys.argv[1], sys.argv[2]
    os.makedirs(dst, exist_ok=True)
    for name in FILES:
        with open(os.path.join(ref, name)) as f:
            text = f.read()
        out = name + ".cpp" if name.endswith(".hlsl") else name
        with open(os.path.join(dst, out), "w") as f:
            f.write(f"// generated from the reference's {name} by oracle/hlsl/hlsl2cpp.py; do not commit\n")
            f.write(rewrite(text))


if __name__ == "__main__":
    main()
