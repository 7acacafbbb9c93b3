"""Build step of the oracle's reference harness (TEST INFRASTRUCTURE ONLY).

Copies the text of the reference's SPAI kernels, exactly as they stand in the
reference tree's src/spai_single_dcu.cpp, into oracle/_ref/ref_spai_kernels.inc
(git-ignored; it never enters this repository's history), so that
oracle/ref_emulate.cpp can compile them unmodified for the host SIMT emulator
(oracle/simt_emu.h).  The kernels are extracted by name: from the template
line above `__global__ void <name>(` through the brace that closes the body.

Run by the oracle Makefile:  python extract_ref_kernels.py <reference-root> <out>
"""
import sys

KERNELS = [
    "computeJ_SSPAIv10", "computeJ2_SSPAIv10",
    "computeIShared_Symbol_SpMMv1", "computeI_Symbol_SpMMv1",
    "computeIShared_iter_Symbol_SpMMv1", "computeI_iter_Symbol_SpMMv1",
    "ComputeTildeACSR_SSPAIv10", "ComputeTildeE_SSPAIv10", "ComputeTildeE2_SSPAIv10",
    "Sol_SSPAIv10", "QR_RShared_SSPAIv10", "modifyData4_SSPAIv10", "modifyData24_SSPAIv10",
]


def extract(lines, name):
    head = None
    for i, line in enumerate(lines):
        if "__global__" in line and f" {name}(" in line:
            head = i
            break
    if head is None:
        raise SystemExit(f"kernel {name} not found")
    start = head - 1 if lines[head - 1].lstrip().startswith("template") else head
    depth, opened = 0, False
    for j in range(head, len(lines)):
        for ch in lines[j]:
            if ch == "{":
                depth += 1
                opened = True
            elif ch == "}":
                depth -= 1
        if opened and depth == 0:
            return start, j
    raise SystemExit(f"kernel {name}: unbalanced braces")


def main():
    root, out = sys.argv[1], sys.argv[2]
    src = f"{root}/src/spai_single_dcu.cpp"
    with open(src, encoding="utf-8", errors="replace") as f:
        lines = f.read().split("\n")
    parts = [f"// Extracted from {src} by oracle/extract_ref_kernels.py; do not edit.\n"]
    for name in KERNELS:
        s, e = extract(lines, name)
        parts.append(f"// ---- {name}: src/spai_single_dcu.cpp:{s + 1}-{e + 1}\n")
        parts.append("\n".join(lines[s:e + 1]) + "\n\n")
    with open(out, "w") as f:
        f.write("".join(parts))


if __name__ == "__main__":
    main()
