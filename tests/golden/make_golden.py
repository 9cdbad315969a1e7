"""Writes tests/golden/sobol_directions.json from the reference itself (run in a
container where the reference is mounted): the direction numbers its generator
tools/sobol_table.py computes, and the table it wrote into shaders/sobol_table.glsl,
which must agree.

    python tests/golden/make_golden.py /path/to/luce-render
"""
import json
import re
import sys
from pathlib import Path


def main(reference: Path) -> None:
    source = (reference / "tools" / "sobol_table.py").read_text()
    # The generator's module body ends by writing the GLSL file; run only the part
    # that defines and evaluates the table.
    body = source[: source.index("lines = [")]
    scope: dict = {}
    exec(compile(body, "sobol_table.py", "exec"), scope)
    generated = [x for row in scope["rows"] for x in row]
    glsl = (reference / "shaders" / "sobol_table.glsl").read_text()
    table = [int(x, 16) for x in re.findall(r"0x([0-9a-f]{8})u", glsl)]
    assert generated == table and len(table) == 128, "generator and shipped table disagree"
    out = Path(__file__).resolve().parent / "sobol_directions.json"
    out.write_text(json.dumps({"source": "tools/sobol_table.py + shaders/sobol_table.glsl",
                               "directions": table}, indent=1) + "\n")
    print(f"wrote {out}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/luce-render")
    main(Path(sys.argv[1]))
