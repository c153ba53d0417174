"""Command-line entry of the package directory:

    python no-three-in-line_b200 tempering --initial state.json --output run --seed 1 [...]

runs the replica-exchange tempering driver (the reference's
``python -m no_three_75.tempering``, src/no_three_75/tempering.py:228-319) with
the same arguments.  The directory name is not a Python identifier, so the
package is loaded under ``no_three_in_line_b200`` first.
"""
from __future__ import annotations

import sys
from pathlib import Path

COMMANDS = ("tempering",)


def _run() -> int:
    root = Path(__file__).resolve().parents[1]
    if str(root) not in sys.path:
        sys.path.insert(0, str(root))
    from __graft_entry__ import load_package

    load_package()
    if len(sys.argv) < 2 or sys.argv[1] not in COMMANDS:
        print(f"usage: python {Path(__file__).resolve().parent.name} {{{','.join(COMMANDS)}}} [arguments]",
              file=sys.stderr)
        return 2
    from no_three_in_line_b200 import tempering

    return tempering.main(sys.argv[2:])


if __name__ == "__main__":
    raise SystemExit(_run())
