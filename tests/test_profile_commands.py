"""Every bench command quoted in profiles/ is accepted by bench.py's own parser,
so each summary names a command that runs on the committed files."""

from __future__ import annotations

import re
import shlex
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def bench_commands():
    for md in sorted((ROOT / "profiles").glob("*.md")):
        for m in re.finditer(r"python bench\.py([^`\n]*)", md.read_text()):
            yield md.name, shlex.split(m.group(1))


def test_profile_commands_parse():
    import bench

    cmds = list(bench_commands())
    assert len(cmds) >= 8
    parser = bench.build_parser()
    for name, argv in cmds:
        try:
            parser.parse_args(argv)
        except SystemExit as e:  # argparse reports unknown or malformed options this way
            raise AssertionError(f"{name}: python bench.py {' '.join(argv)}") from e
