"""The in-tree build (luce_render_b200/build.py) on the host: an object compiled by another
step since the last link (newer than the library) is linked in, although nothing needed
compiling in this call."""
import os
import shutil
import time

import pytest

from luce_render_b200 import build


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="needs nvcc")
def test_object_newer_than_library_is_linked():
    build.build()  # up to date first
    objects = [build.BUILD / (src.name + ".o") for src in build.sources()]
    assert all(o.exists() for o in objects)
    # An object newer than the library stands for one compiled by another step since the
    # last link (both in the past, so the new link is newer than every object).
    now = time.time()
    os.utime(build.LIBRARY, (now - 100.0, now - 100.0))
    os.utime(objects[0], (now - 50.0, now - 50.0))
    before = build.LIBRARY.stat().st_mtime
    build.build()
    after = build.LIBRARY.stat().st_mtime
    assert after > before
    # Nothing newer now: no second link.
    build.build()
    assert build.LIBRARY.stat().st_mtime == after
