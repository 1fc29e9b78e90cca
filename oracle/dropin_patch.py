"""Applies the maintainer's Backend::B200 patch to a COPY of the reference tree.
TEST INFRASTRUCTURE ONLY.

    python3 dropin_patch.py <build dir holding copies of the reference include/ and src/>

The two edits INTEGRATION.md shows a maintainer making to plug this backend
into the reference library, applied to the copy in the build directory (never
to the reference tree itself):

* include/processorconfiguration.h: one enumerator, ``B200``, after ``CPU`` in
  ``enum class Backend`` (existing values keep their numbers);
* src/core/processor.cpp: ``#include "b200_backend.h"`` and, in
  ``Processor::Impl::createBackend`` (processor.cpp:38-50), a case that makes
  an ``ope::B200Backend``.

Fails loudly if either anchor is not found, rather than building an unpatched
library.
"""
from __future__ import annotations

import os
import re
import sys


def patch(build: str) -> None:
    hdr = os.path.join(build, "include", "processorconfiguration.h")
    with open(hdr) as f:
        s = f.read()
    s2, n = re.subn(r"(enum\s+class\s+Backend\s*\{[^}]*?\bCPU\b)(\s*\})", r"\1,\n\tB200\2", s, count=1)
    if n != 1:
        raise SystemExit(f"{hdr}: enum class Backend {{ ..., CPU }} not found")
    with open(hdr, "w") as f:
        f.write(s2)

    src = os.path.join(build, "src", "core", "processor.cpp")
    with open(src) as f:
        s = f.read()
    s2, n1 = re.subn(r'(#include\s+"\.\./backends/cpu/cpu_backend\.h"\s*\n)', r'\1#include "b200_backend.h"\n', s,
                     count=1)
    s3, n2 = re.subn(r"(\n(\s*)case\s+Backend::CPU:\s*\n\s*this->backend\s*=\s*std::make_unique<CpuBackend>\(\);\s*\n"
                     r"\s*break;\s*\n)",
                     r"\1\2case Backend::B200:\n\2\tthis->backend = std::make_unique<B200Backend>();\n\2\tbreak;\n",
                     s2, count=1)
    if n1 != 1 or n2 != 1:
        raise SystemExit(f"{src}: createBackend anchors not found")
    with open(src, "w") as f:
        f.write(s3)


if __name__ == "__main__":
    patch(sys.argv[1])
