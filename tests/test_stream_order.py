"""Every copy and zero fill of engine memory is ordered on the engine's stream.

The engine launches on a stream created with cudaStreamNonBlocking, which the
legacy default stream does not synchronise with.  A plain cudaMemcpy or
cudaMemset runs on the legacy stream, so it can overtake, or be overtaken by,
the engine's kernels and its cudaMemsetAsync zero fills: a host upload into a
freshly allocated buffer could be wiped by the buffer's pending zero fill.
The sources therefore copy through Engine::h2d / Engine::d2h (cudaMemcpyAsync
on the engine stream, then a stream synchronise) and fill with
cudaMemsetAsync on that stream.  This reads the sources; no GPU is needed.
"""

from __future__ import annotations

import re

from tests.conftest import ROOT

LEGACY = re.compile(
    r"\b(cudaMemcpy|cudaMemset|cudaMemcpy2D|cudaMemcpyToSymbol|cudaMemcpyFromSymbol|"
    r"cudaMemcpyPeer)\s*\("
)


def _code(text: str) -> str:
    text = re.sub(r'"(?:[^"\\\n]|\\.)*"', '""', text)  # string literals
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def test_no_legacy_stream_copies_in_engine_sources():
    hits = []
    for path in sorted((ROOT / "beads_b200" / "csrc").glob("*")):
        if path.suffix not in (".cu", ".cuh", ".cpp", ".hpp"):
            continue
        for no, line in enumerate(_code(path.read_text()).splitlines(), 1):
            if LEGACY.search(line):
                hits.append(f"{path.name}:{no}: {line.strip()}")
    assert not hits, "\n".join(hits)


def test_async_copies_name_a_stream():
    # cudaMemcpyAsync / cudaMemsetAsync without an explicit stream argument
    # default to stream 0, the legacy stream.
    calls = re.compile(r"\b(cudaMemcpyAsync|cudaMemsetAsync|cudaMemcpy2DAsync)\s*\(")
    bad = []
    for path in sorted((ROOT / "beads_b200" / "csrc").glob("*")):
        if path.suffix not in (".cu", ".cuh", ".cpp", ".hpp"):
            continue
        text = _code(path.read_text())
        for m in calls.finditer(text):
            depth, j = 0, m.end() - 1
            while j < len(text):
                if text[j] == "(":
                    depth += 1
                elif text[j] == ")":
                    depth -= 1
                    if depth == 0:
                        break
                j += 1
            args = text[m.end():j]
            last = args.rsplit(",", 1)[-1].strip()
            if last in ("0", "nullptr", "NULL", "cudaStreamLegacy") or args.count(",") < 3:
                bad.append(f"{path.name}: {m.group(1)}({args.strip()[:80]})")
    assert not bad, "\n".join(bad)
