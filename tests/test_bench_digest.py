"""bench.py's digest of the kernel sources, which says whether the committed
ncu figures were captured from the code being benchmarked: it follows code
changes and ignores comments and blank lines."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_code_lines_drop_comments_and_blank_lines():
    src = "int a = 1;  // note\n\n// a comment line\n  b += a;   \nfloat f(float /*x*/);\n"
    assert bench._code_lines(src) == "int a = 1;\n  b += a;\nfloat f(float /*x*/);"


def test_digest_follows_code_and_ignores_comments(tmp_path, monkeypatch):
    csrc = tmp_path / "dpa_b200" / "csrc"
    csrc.mkdir(parents=True)
    for name in bench.KERNEL_SOURCES:
        (csrc / name).write_text(f"// {name}\nint x_{name.replace('.', '_')} = 1;\n")
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    base = bench.kernel_sources_digest()
    first = csrc / bench.KERNEL_SOURCES[0]
    first.write_text(first.read_text() + "// a new comment\n\n")
    assert bench.kernel_sources_digest() == base
    first.write_text(first.read_text() + "int y = 2;\n")
    assert bench.kernel_sources_digest() != base


def test_kernel_sources_hold_no_double_slash_in_string_literals():
    # _code_lines cuts at the first "//" of a line, which would also cut a
    # string literal holding one.
    for name in bench.KERNEL_SOURCES:
        for line in (ROOT / "dpa_b200" / "csrc" / name).read_text().splitlines():
            code = line.split("//", 1)[0]
            assert code.count('"') % 2 == 0, (name, line)
