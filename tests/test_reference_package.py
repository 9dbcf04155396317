"""The reference's own Python package (python/src/unround of JPEG-Unround), unchanged, driving this
build's library through UNROUND_LIBRARY, as a user of the reference switches to it: its ctypes
bindings of every function it declares load against libunround_capi.so; the version, the
settings it holds, the reading of a JPEG file's coefficients (the C layer it reaches through the
same library), JFIF's colour conversions and the projection of a picture onto a file's intervals
(host binary64) come out bit for bit as this repository's package gives them; and a solve without
a CUDA device fails with the reference's own error, status INTERNAL, as this build refuses to run
on the host.

The reference package runs in a child process (its package name is this repository's too), with
its annotations postponed: on this image's Python 3.12 its modules name their own classes in
annotations before the classes exist. It reads the reference checkout, so the test runs only
where the checkout is (UNROUND_REFERENCE names it); the GPU machines have none."""

import io
import json
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import numpy as np
import pytest

REFERENCE = Path(os.environ.get("UNROUND_REFERENCE") or "/root/reference")
PACKAGE = REFERENCE / "python" / "src"

pytestmark = pytest.mark.skipif(not (PACKAGE / "unround" / "native.py").is_file(),
                                reason="the reference checkout is not on this machine")

CHILD = textwrap.dedent('''
    import importlib.abc, importlib.machinery, importlib.util, json, sys
    import numpy as np

    source_root = sys.argv[1]

    class Postponed(importlib.machinery.SourceFileLoader):
        def source_to_code(self, data, path, *, _optimize=-1):
            return compile(b"from __future__ import annotations\\n" + data, path, "exec", dont_inherit=True)

    class Finder(importlib.abc.MetaPathFinder):
        def find_spec(self, name, path=None, target=None):
            if name != "unround" and not name.startswith("unround."):
                return None
            spec = importlib.machinery.PathFinder.find_spec(name, path or [source_root])
            if spec is not None and spec.origin and spec.origin.endswith(".py"):
                spec.loader = Postponed(spec.name, spec.origin)
            return spec

    sys.meta_path.insert(0, Finder())
    import unround
    from unround import jpegio, native
    from unround.settings import PdhgOptions, Settings

    work = sys.argv[2]
    data = np.load(work + "/inputs.npz")
    jpeg = bytes(data["jpeg"])
    out = {"module": unround.__file__, "version": native.version()}
    settings = Settings(method="tv", pdhg=PdhgOptions(iterations=40, tolerance=0.0, record_every=5))
    out["held"] = list(native.held_options(settings))
    image = jpegio.read(jpeg)
    arrays = {f"levels_{k}": c.coefficients for k, c in enumerate(image.components)}
    arrays.update({f"table_{k}": np.asarray(c.quant_table) for k, c in enumerate(image.components)})
    arrays["rgb"] = native.to_rgb(data["ycbcr"])
    arrays["ycbcr"] = native.to_ycbcr(data["rgb"])
    projected = native.project(data["picture"], jpeg)
    arrays["projected"] = np.asarray(projected.picture)
    try:
        native.solve(image, settings)
        out["solve"] = "solved"
    except native.UnroundError as error:
        out["solve"] = {"type": type(error).__module__ + "." + type(error).__name__,
                        "status": int(error.status), "message": str(error)}
    np.savez(work + "/outputs.npz", **arrays)
    print(json.dumps(out))
''')


def test_the_reference_package_drives_this_library(tmp_path):
    from PIL import Image

    from unround import jpegio, native, synthetic

    rgb = synthetic.colour(45, 62, quality=50, seed=81, noise=2).samples
    stream = io.BytesIO()
    Image.fromarray(np.clip(rgb, 0, 255).astype(np.uint8)).save(stream, format="JPEG", quality=60, subsampling=2)
    jpeg = stream.getvalue()
    picture = np.clip(rgb + np.random.default_rng(3).normal(0, 4, rgb.shape), 0, 255)
    ycbcr = synthetic.ycbcr(rgb)
    np.savez(tmp_path / "inputs.npz", jpeg=np.frombuffer(jpeg, dtype=np.uint8), rgb=rgb, ycbcr=ycbcr, picture=picture)

    environment = {**os.environ, "UNROUND_LIBRARY": native.library_path(), "PYTHONPATH": ""}
    run = subprocess.run([sys.executable, "-c", CHILD, str(PACKAGE), str(tmp_path)], env=environment,
                         capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr[-3000:]
    told = json.loads(run.stdout.strip().splitlines()[-1])
    got = np.load(tmp_path / "outputs.npz")

    # It is the reference's package that ran, on this build's library.
    assert Path(told["module"]).resolve().is_relative_to(PACKAGE.resolve())
    assert told["version"] == native.version() and "B200" in told["version"]
    from unround.settings import PdhgOptions, Settings

    ours = native.held_options(Settings(method="tv", pdhg=PdhgOptions(iterations=40, tolerance=0.0, record_every=5)))
    assert told["held"] == list(ours)
    image = jpegio.read(jpeg)
    for k, component in enumerate(image.components):
        np.testing.assert_array_equal(got[f"levels_{k}"], component.coefficients)
        np.testing.assert_array_equal(got[f"table_{k}"], np.asarray(component.quant_table))
    np.testing.assert_array_equal(got["rgb"], native.to_rgb(ycbcr))
    np.testing.assert_array_equal(got["ycbcr"], native.to_ycbcr(rgb))
    np.testing.assert_array_equal(got["projected"], np.asarray(native.project(picture, jpeg).picture))
    solve = told["solve"]
    assert isinstance(solve, dict), solve  # no CUDA device here: the solve is refused, not run on the host
    assert solve["type"] == "unround.native.UnroundError"
    assert solve["status"] == int(native.Status.INTERNAL) and "CUDA" in solve["message"]
