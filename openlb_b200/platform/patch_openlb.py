#!/usr/bin/env python3
"""Prepare an OpenLB source tree that knows Platform::GPU_B200.

    python patch_openlb.py --openlb /path/to/openlb --out BUILD_DIR

Copies OpenLB's src/ to BUILD_DIR/src and makes the five additions a
maintainer would commit to adopt the platform (the reference's platform seam):

  src/core/platform/platform.h       the GPU_B200 tag of enum struct Platform
                                     (:35-39) and its isPlatformCPU case
  src/core/platform/dispatch.h       a GPU_B200 case beside every GPU_CUDA case
                                     of the dispatch switches (:40-132)
  src/communication/loadBalancer.h   GPU_B200 as the default platform when
                                     built with PLATFORM_GPU_B200 (:102-118)
  src/core/blockLattice.h            include of olb_b200_platform.h (the
                                     specialisations) when PLATFORM_GPU_B200
  src/olb3D.h                        include of olb_b200_dynamics.h (which
                                     dynamics the device implements; it names
                                     aliases declared after blockLattice.h)

Every edit is anchored on text of the original files; if an anchor is missing
(a different OpenLB version) the script stops with an error instead of
producing a half-patched tree.  Examples are compiled from their original
location, unmodified, against BUILD_DIR/src with -DPLATFORM_GPU_B200.
"""
from __future__ import annotations

import argparse
import re
import shutil
import sys
from pathlib import Path


class AnchorMissing(RuntimeError):
    pass


def _edit(path: Path, fn) -> None:
    text = path.read_text()
    new = fn(text)
    if new == text:
        raise AnchorMissing(f"{path}: nothing changed")
    path.write_text(new)


def platform_h(text: str) -> str:
    anchor = "  GPU_CUDA, /// GPU using CUDA\n"
    if anchor not in text:
        raise AnchorMissing("platform.h: GPU_CUDA enumerator")
    text = text.replace(anchor, anchor + "  GPU_B200, /// NVIDIA B200 through libolb_b200 (C ABI)\n", 1)
    # isPlatformCPU: the B200 platform keeps host copies but computes on the device
    m = re.search(r"(constexpr bool isPlatformCPU\(Platform platform\) \{.*?)(\n  default:)", text, re.S)
    if not m:
        raise AnchorMissing("platform.h: isPlatformCPU switch")
    case = "\n#ifdef PLATFORM_GPU_B200\n  case Platform::GPU_B200:\n    return false;\n#endif"
    return text[:m.end(1)] + case + text[m.end(1):]


def dispatch_h(text: str) -> str:
    """Duplicate every `#ifdef PLATFORM_GPU_CUDA ... #endif` case block of the
    dispatch switches for GPU_B200."""
    pattern = re.compile(r"#ifdef PLATFORM_GPU_CUDA\n(.*?)#endif\n", re.S)
    count = 0

    def dup(m):
        nonlocal count
        count += 1
        body = m.group(1).replace("GPU_CUDA", "GPU_B200")
        return m.group(0) + "#ifdef PLATFORM_GPU_B200\n" + body + "#endif\n"

    out = pattern.sub(dup, text)
    if count != 3:
        raise AnchorMissing(f"dispatch.h: expected 3 GPU_CUDA cases, found {count}")
    return out


def load_balancer_h(text: str) -> str:
    anchor = "    #ifdef PLATFORM_GPU_CUDA\n      return Platform::GPU_CUDA;\n"
    if anchor not in text:
        raise AnchorMissing("loadBalancer.h: default platform")
    return text.replace(anchor, "    #ifdef PLATFORM_GPU_B200\n      return Platform::GPU_B200;\n    #endif\n"
                        + anchor, 1)


def block_lattice_h(text: str) -> str:
    idx = text.rstrip().rfind("#endif")
    if idx < 0:
        raise AnchorMissing("blockLattice.h: include guard")
    return text[:idx] + "#ifdef PLATFORM_GPU_B200\n#include \"olb_b200_platform.h\"\n#endif\n\n" + text[idx:]


def olb3d_h(text: str) -> str:
    # olb3D.h is a plain list of includes (no guard): append after the last one
    anchor = "#include <uq/uq.h>\n"
    if anchor not in text:
        raise AnchorMissing("olb3D.h: last include")
    return text.replace(anchor, anchor + "\n#ifdef PLATFORM_GPU_B200\n#include \"olb_b200_dynamics.h\"\n#endif\n", 1)


EDITS = {
    "core/platform/platform.h": platform_h,
    "core/platform/dispatch.h": dispatch_h,
    "communication/loadBalancer.h": load_balancer_h,
    "core/blockLattice.h": block_lattice_h,
    "olb3D.h": olb3d_h,
}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--openlb", required=True, help="OpenLB source tree (read only)")
    ap.add_argument("--out", required=True, help="build directory for the patched copy")
    args = ap.parse_args(argv)
    src = Path(args.openlb) / "src"
    if not (src / "olb.h").exists():
        print(f"patch_openlb: {src} is not an OpenLB source tree", file=sys.stderr)
        return 2
    out = Path(args.out)
    dst = out / "src"
    if dst.exists():
        shutil.rmtree(dst)
    shutil.copytree(src, dst)
    for rel, fn in EDITS.items():
        _edit(dst / rel, fn)
    (out / "PATCHED").write_text("".join(f"{rel}\n" for rel in EDITS))
    return 0


if __name__ == "__main__":
    sys.exit(main())
