"""The C interface without a GPU: the library loads, is of ABI version 5, exports every function
include/*.h declares with the reference's structure layouts, parses the command line's options
as the reference does (names, ranges, refusals all at once, values held), and refuses to solve
loudly where there is no CUDA device (there is no CPU fallback)."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from unround import native, synthetic

INCLUDE = Path(__file__).resolve().parents[1] / "include"


def _declared() -> list[str]:
    names = []
    for header in INCLUDE.rglob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        names += re.findall(r"\b(unround_\w+)\s*\(", text)
    return sorted(set(names))


def test_exports_every_declared_function():
    library = ctypes.CDLL(native.library_path())
    names = _declared()
    assert "unround_solve" in names and "unround_settings_new" in names
    missing = [name for name in names if not hasattr(library, name)]
    assert missing == []


def test_version_and_layouts():
    assert native._library().unround_abi_version() == 5
    assert "unround" in native.version()
    assert ctypes.sizeof(native._Record) == 64
    assert ctypes.sizeof(native._Component) == 152
    assert native._Component.quant_table.offset == 24
    assert ctypes.sizeof(native._Input) == 24
    assert native._Input.components.offset == 16


def test_default_settings_held():
    held = native.held_options()
    assert "--method=tgv" in held and "--alpha1=1" in held and "--alpha0=2" in held
    assert "--mu=rule" in held and "--mu-scale=9" in held and "--flat-weight=0.1" in held
    assert "--record-every=10" in held and "--relaxation=1.9" in held and "--step-product=0.99" in held


def test_options_round_trip():
    given = ["--method", "tv", "--alpha", "0.5", "--mu", "0.01,0.02,0.03", "--centres=mmse", "--flat-dc", "any",
             "--iterations", "40", "--tolerance", "0", "--no-weight-scaling", "--channels", "apart"]
    held = native.held_options(given)
    again = native.held_options(held)
    assert held == again
    assert "--mu=0.01,0.02,0.03" in held and "--flat-dc=any" in held and "--no-weight-scaling" in held


@pytest.mark.parametrize(
    "options, fragment",
    [
        (["--mu", "-1"], "--mu is at least 0"),
        (["--method", "nope"], "--method is one of"),
        (["--relaxation", "2"], "--relaxation is between 0 and 2"),
        (["--alpha", "1", "--alpha", "2"], "--alpha is given twice"),
        (["--bogus"], "--bogus is not an option"),
        (["--method", "tv", "--partial-radius", "3"], "TGV's alone"),
        (["--partial-tolerance", "1"], "needs --partial-radius"),
        (["--mu", "1,2", "--slack", "1,2,3"], "one value for every component or one for each"),
        (["--iterations"], "needs a value"),
    ],
)
def test_refusals(options, fragment):
    with pytest.raises(native.UnroundError) as raised:
        native.held_options(options)
    assert raised.value.status == native.Status.OPTIONS
    assert fragment in raised.value.message


def test_every_refusal_at_once():
    with pytest.raises(native.UnroundError) as raised:
        native.held_options(["--mu", "-1", "--relaxation", "3"])
    assert "--mu" in raised.value.message and "--relaxation" in raised.value.message


def test_file_paths_refuse_what_they_cannot_read():
    # A JPEG file cut after its first marker holds no image: READ, before any device is needed.
    with pytest.raises(native.UnroundError) as raised:
        native.decode(b"\xff\xd8\xff")
    assert raised.value.status == native.Status.READ
    # Nor can a picture be projected onto the intervals of a file that holds no image.
    with pytest.raises(native.UnroundError) as raised:
        native.project(np.zeros((8, 8)), b"\xff\xd8\xff\xd9")
    assert raised.value.status == native.Status.READ


def test_colour_conversions_invert():
    rng = np.random.default_rng(0)
    rgb = rng.uniform(0, 255, size=(5, 7, 3))
    back = native.to_rgb(native.to_ycbcr(rgb))
    np.testing.assert_allclose(back, rgb, atol=1e-10)


def test_solve_fails_loudly_without_a_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    image = synthetic.grey(16, 16, seed=0).image
    with pytest.raises(native.UnroundError) as raised:
        native.solve(image, ["--method", "tv", "--iterations", "2"])
    assert raised.value.status == native.Status.INTERNAL
    assert "CUDA" in raised.value.message


@pytest.mark.parametrize("orientation", range(9))
def test_oriented_turns_as_exif_says(orientation):
    # EXIF 2.3 tag 0x0112 (the reference's rust/unround/src/orientation.rs): 0 or 1 as stored,
    # 2 mirrored, 3 half round, 4 flipped, 5 transposed, 6 a quarter clockwise, 7 transversed,
    # 8 a quarter anticlockwise.
    picture = np.arange(3 * 5 * 2, dtype=np.float64).reshape(3, 5, 2)
    expected = {
        0: picture, 1: picture, 2: picture[:, ::-1], 3: picture[::-1, ::-1], 4: picture[::-1],
        5: picture.transpose(1, 0, 2), 6: np.rot90(picture, -1), 7: np.rot90(picture, -1)[::-1],
        8: np.rot90(picture, 1),
    }[orientation]
    np.testing.assert_array_equal(native.oriented(picture, orientation), expected)
    np.testing.assert_array_equal(native.oriented(picture[..., 0], orientation), expected[..., 0])


def test_oriented_refuses_what_is_no_orientation():
    with pytest.raises(native.UnroundError):
        native.oriented(np.zeros((2, 3)), 9)


def test_the_c_layer_s_metadata_and_the_profile_check():
    from unround import jpegio

    assert jpegio.abi_version() == jpegio.ABI_VERSION
    assert "JPEG reader" in jpegio.libjpeg_version() and "zlib" in jpegio.libpng_version()
    assert jpegio.check_icc(b"\0" * 200, 3) is not None  # no 'acsp', no length


def test_the_command_line_is_outside_this_build():
    assert native.main(["--help"]) == 3


def _copy_in_child(out) -> None:
    data = np.arange(3_000_000, dtype=np.float64)
    copied = native._copy(data.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), (1000, 3000))
    out.put(bool(np.array_equal(copied.reshape(-1), data)))


@pytest.mark.filterwarnings("ignore:This process .* is multi-threaded:DeprecationWarning")
def test_large_copies_in_parts_and_after_fork():
    """A result's large arrays are copied on the host's threads, in parts, exactly; a process forked
    after the copying threads exist makes its own (the parent's do not exist in the child)."""
    import multiprocessing as mp

    data = np.arange(5_000_000, dtype=np.float64)  # 40 MB: copied in parts
    copied = native._copy(data.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), (5000, 1000))
    assert copied.shape == (5000, 1000) and np.array_equal(copied.reshape(-1), data)
    assert copied.ctypes.data != data.ctypes.data
    context = mp.get_context("fork")
    out = context.Queue()
    child = context.Process(target=_copy_in_child, args=(out,))
    child.start()
    child.join(timeout=60)
    assert child.exitcode == 0 and out.get(timeout=5) is True
