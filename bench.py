"""Throughput of the TV/TGV primal-dual reconstruction on B200, in megapixel-iterations per second.

The workload is the reconstruction of a 4032x3024 YCbCr 4:2:0 picture (seeded synthetic
piecewise-smooth picture per RGB channel with Gaussian noise sigma 3, quality 75 standard
tables) by TGV with alpha0 = 2, alpha1 = 1, 500 iterations, all three planes, binary32 state.
A step is one full solve of it (500 iterations).

  value  the iteration loop alone with the state resident in HBM: device time of K steps by CUDA
         events on the solve's stream (unround_b200_measure), max over ranks; the state (~3 GB)
         is larger than L2, so no flush is needed between iterations.
  e2e    the same metric through the drop-in call (unround.native.solve -> unround_solve) with
         host arrays: levels copied in, the binary64 result copied out, every step.

Beside them, outside the timed regions: cpu_baseline (the reference's C++ solver on the host
cores, run first: the median of five bounded samples with every thread and of three with one,
and one whole solve of the workload), parity (the device's result against that whole solve), records (the
cost of a record every 10 iterations, the reference's default), mix (the batched 64-picture mix
against the same pictures one at a time, with the ceiling the image-at-a-time path's share of
the HBM peak leaves).

With --gpus N (under torchrun) each rank solves its own picture (images are independent units,
no data-path collective): weak scaling, value = all ranks' pixel-iterations / max time.
--impl reference times the reference's own C++ solver (oracle/_ref) on the host cores instead.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
HEIGHT, WIDTH, ITERATIONS = 3024, 4032, 500
OPTIONS = ["--method", "tgv", "--alpha1", "1", "--alpha0", "2", "--iterations", str(ITERATIONS), "--tolerance", "0",
           "--record-every", "0"]
METRIC = "TGV PDHG Mpx*iter/s on 1 B200 (4032x3024 YCbCr 4:2:0, 500 iterations)"
UNIT = "Mpx*iter/s"
# Algorithmic bytes per sample-iteration of the fused TGV iteration in binary32, 4:2:0
# (8 fields read and written, 4 B each, and the int16 levels: (2 + 2*2/4) / 3 = 1 B per sample).
ALGORITHMIC_BYTES = 65.0
# The dual kernel alone: x~, x, w(2), p(2), r(3) read and x, w, p, r written.
DUAL_BYTES = 17 * 4.0


def _rank() -> tuple[int, int, int]:
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def _peaks() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def _copy_gbs() -> float:
    """The device's copy bandwidth on this box, now: a 2 GiB device-to-device copy (read and
    write counted), the best of 10 timed by CUDA events after 3 warm-up copies. Reported beside
    the peak, so a fraction can be read against the same box and clocks."""
    import torch

    n = (2 << 30) // 4
    source = torch.empty(n, dtype=torch.float32, device="cuda")
    target = torch.empty_like(source)
    source.fill_(1.0)
    for _ in range(3):
        target.copy_(source)
    best = None
    for _ in range(10):
        begin, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        begin.record()
        target.copy_(source)
        end.record()
        end.synchronize()
        ms = begin.elapsed_time(end)
        best = ms if best is None else min(best, ms)
    del source, target
    torch.cuda.empty_cache()
    return 2 * n * 4 / (best / 1e3) / 1e9


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int) -> None:
        self.device = device
        self.samples: list[list[str]] = []
        self._process: subprocess.Popen | None = None
        self._thread: threading.Thread | None = None

    def __enter__(self) -> Clocks:
        try:
            self._process = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._thread = threading.Thread(target=self._read, daemon=True)
            self._thread.start()
        except OSError:
            self._process = None
        # nvidia-smi takes a moment to start: the timed region begins once it samples (3 s at
        # most), so that a short region is sampled too.
        for _ in range(60):
            if self.samples or self._process is None or self._process.poll() is not None:
                break
            time.sleep(0.05)
        return self

    def _read(self) -> None:
        assert self._process is not None and self._process.stdout is not None
        for line in self._process.stdout:
            self.samples.append([part.strip() for part in line.split(",")])

    def __exit__(self, *_: object) -> None:
        if self._process is not None:
            self._process.terminate()
            self._process.wait(timeout=5)
        if self._thread is not None:
            self._thread.join(timeout=2)

    def summary(self) -> dict:
        """The median SM clock under load -- over the samples drawing at least half the most
        power drawn in the region, so that the idle moments around a short timed region (the
        host's set-up, the sampler's start) do not count -- the highest clock, and the throttle
        reasons seen in any sample."""
        def number(text: str) -> float | None:
            try:
                return float(text)
            except ValueError:
                return None

        rows = [s for s in self.samples if len(s) >= 9]
        readings = [(number(s[1]), number(s[3])) for s in rows]
        most = max((w for _, w in readings if w is not None), default=None)
        loaded = [m for m, w in readings if m is not None and (most is None or (w is not None and w >= 0.5 * most))]
        top = [t for t in (number(s[2]) for s in rows) if t is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in rows for k in range(4) if s[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(top) if top else None,
                "reasons": reasons, "samples": len(self.samples), "samples_under_load": len(loaded),
                "power_w_max": most}


def _workload(seed: int):
    from unround import synthetic

    return synthetic.colour(HEIGHT, WIDTH, quality=75, seed=seed, noise=3.0).image


def _components(image):
    return [(c.coefficients, c.quant_table.reshape(64), c.h_samp_factor, c.v_samp_factor) for c in image.components]


def _reference_seconds(image, threads: int, sample: int, repeats: int) -> list[float]:
    """Seconds of `sample` iterations of the reference's solver on the picture with `threads`
    host threads, `repeats` times: each a solve of 1 + sample iterations less one of 1 iteration
    (the host model, the start and the first iteration differenced out)."""
    from oracle import reference

    def run(iterations: int) -> float:
        options = [*OPTIONS[:6], "--iterations", str(iterations), "--tolerance", "0", "--record-every", "0",
                   "--threads", str(threads)]
        began = time.perf_counter()
        reference.solve(image.height, image.width, int(image.color_space), _components(image), options)
        return time.perf_counter() - began

    return [max(run(1 + sample) - run(1), 1e-9) for _ in range(repeats)]


def _reference_arm(args: argparse.Namespace, rank: int) -> None:
    """The reference's own C++ solver on the host cores: each step a bounded sample of the
    workload (two iterations of the same picture, setup excluded by differencing)."""
    if rank != 0:
        return
    from oracle import reference

    if not reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libunround_ref.so is not built"}))
        return
    image = _workload(seed=0)
    threads = os.cpu_count() or 1
    sample = 2
    _reference_seconds(image, threads, 1, args.warmup)
    per_step = statistics.median(_reference_seconds(image, threads, sample, args.steps))
    pixels = HEIGHT * WIDTH
    value = pixels * sample / per_step / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded piecewise-smooth + noise sigma 3)",
        "config": {"workload": "tgv-colour-4032x3024-420", "iterations_per_step": sample,
                   "sample": f"{sample} iterations of the full picture per step (setup differenced out)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{sample} iterations of the 4032x3024 4:2:0 TGV workload, {threads} threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def _cpu_baseline(image) -> tuple[dict | None, object]:
    """The reference's solver on the host cores, a bounded sample: two iterations (setup
    differenced out), the median of five -- the reference arm's estimator, since a solve's setup
    (the host model, the first touch of its arrays) varies by more than two iterations take, so
    that the best of a few samples overstates the rate -- with every host thread and with one
    (median of three); then one whole
    solve of the workload (500 iterations, every thread), timed, whose canvas is the checker of
    the device's result (the line's parity). Run before the process touches the GPU, so that
    nothing of the GPU's side (its driver threads, pinned host memory) competes with it.
    Returns the baseline and the reference's solve (None where oracle/_ref is not built)."""
    from oracle import reference

    if not reference.available():
        return None, None
    threads = os.cpu_count() or 1
    sample, repeats = 2, 5
    _reference_seconds(image, threads, 1, 1)  # the library's pages and the picture's arrays warmed
    samples = _reference_seconds(image, threads, sample, repeats)
    middle = statistics.median(samples)
    one = statistics.median(_reference_seconds(image, 1, sample, 3))
    began = time.perf_counter()
    whole = reference.solve(image.height, image.width, int(image.color_space), _components(image),
                            [*OPTIONS, "--threads", str(threads)])
    whole_seconds = time.perf_counter() - began
    pixels = HEIGHT * WIDTH
    return {"value": pixels * sample / middle / 1e6, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{sample} iterations of the 4032x3024 4:2:0 TGV workload (setup differenced out), "
                      f"median of {repeats}, {threads} threads",
            "best_of_samples": pixels * sample / min(samples) / 1e6,
            "one_thread": {"value": pixels * sample / one / 1e6, "unit": UNIT, "cores": 1,
                           "sample": f"{sample} iterations, median of 3, 1 thread"},
            "whole_solve": {"seconds": whole_seconds, "iterations": ITERATIONS, "cores": threads,
                            "value": pixels * ITERATIONS / whole_seconds / 1e6, "unit": UNIT,
                            "note": "one solve of 500 iterations with the host model and the start"}}, whole


def _parity(decoded, theirs, image) -> dict:
    """The device's result of the workload against the reference's solve of it (binary64):
    canvas relative L2 and max |difference| (0..255), the share of 8-bit output samples that are
    identical, and whether every coefficient lies inside its interval in binary64."""
    import numpy as np

    from unround import native

    difference = decoded.canvas - theirs.canvas
    rounded = lambda x: np.clip(np.sign(x) * np.floor(np.abs(x) + 0.5), 0, 255)  # noqa: E731
    theirs_picture = native.to_rgb(theirs.canvas[:, : image.height, : image.width])
    inside = all(bool(np.all(c >= p.lower) and np.all(c <= p.upper))
                 for c, p in zip(decoded.coefficients, decoded.problems))
    return {"against": "the reference's solver (oracle/_ref, binary64), same picture and options",
            "rel_l2": float(np.linalg.norm(difference) / np.linalg.norm(theirs.canvas)),
            "max_abs": float(np.abs(difference).max()),
            "same_8bit": float(np.mean(rounded(decoded.picture) == rounded(theirs_picture))),
            "inside_intervals": inside, "bar": {"rel_l2": 1e-4, "max_abs": 2e-3, "same_8bit": 0.999}}


def _traffic() -> float | None:
    """DRAM bytes per launch of the dual kernel at this workload, from the committed ncu summary."""
    path = ROOT / "profiles" / "traffic.json"
    try:
        return float(json.loads(path.read_text())["dual_kernel_bytes_per_launch_4032x3024_420"])
    except (OSError, KeyError, ValueError):
        return None


def _jpeg_file(seed: int) -> bytes:
    """The workload's picture (the same generator, size and noise) as a JPEG file, quality 75, 4:2:0,
    written by Pillow's libjpeg-turbo: the file path's input."""
    import io

    import numpy as np
    from PIL import Image

    from unround import synthetic

    rgb = synthetic.colour(HEIGHT, WIDTH, quality=75, seed=seed, noise=3.0).samples
    buffer = io.BytesIO()
    Image.fromarray(np.clip(np.rint(rgb), 0, 255).astype(np.uint8)).save(buffer, format="JPEG", quality=75,
                                                                         subsampling=2)
    return buffer.getvalue()


def _call_file(data: bytes) -> int:
    """One solve of a JPEG file through unround_decode: the file's bytes in (the coefficients read
    on the host by the library), the binary64 canvas and picture out and read on the host."""
    import ctypes

    import numpy as np

    from unround import native

    library = native._library()
    settings = native._Settings(OPTIONS)
    result = ctypes.c_void_p()
    message = ctypes.create_string_buffer(4096)
    status = library.unround_decode(data, len(data), settings.handle, native._OBSERVER(), None, ctypes.byref(result),
                                    message, 4096)
    if status != 0:
        raise RuntimeError(message.value.decode())
    try:
        c, h, w = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        canvas = np.ctypeslib.as_array(library.unround_result_canvas(result, ctypes.byref(c), ctypes.byref(h),
                                                                     ctypes.byref(w)),
                                       shape=(c.value * h.value * w.value,))
        ph, pw, pc = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        picture = np.ctypeslib.as_array(library.unround_result_picture(result, ctypes.byref(ph), ctypes.byref(pw),
                                                                       ctypes.byref(pc)),
                                        shape=(ph.value * pw.value * pc.value,))
        if not (np.isfinite(canvas[:: max(1, canvas.size // 4096)]).all()
                and np.isfinite(picture[:: max(1, picture.size // 4096)]).all()):
            raise RuntimeError("the result holds values that are not finite")
        return canvas.nbytes + picture.nbytes
    finally:
        library.unround_result_free(result)


def _call(image, options: list[str] | None = None) -> int:
    """One solve through the C interface, as a C or cgo caller makes it: unround_solve on host
    arrays (levels in; the binary64 canvas, coefficients and RGB picture out, into the result),
    then the canvas and the picture read on the host. Returns the result's bytes copied from the
    device (the picture is made on the device and copied like the canvas). The options are the
    workload's unless given."""
    import ctypes

    import numpy as np

    from unround import native

    library = native._library()
    settings = native._Settings(OPTIONS if options is None else options)
    given, kept = native._input_of(image)
    result = ctypes.c_void_p()
    message = ctypes.create_string_buffer(4096)
    status = library.unround_solve(ctypes.byref(given), settings.handle, native._OBSERVER(), None,
                                   ctypes.byref(result), message, 4096)
    if status != 0:
        raise RuntimeError(message.value.decode())
    try:
        c, h, w = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        pointer = library.unround_result_canvas(result, ctypes.byref(c), ctypes.byref(h), ctypes.byref(w))
        canvas = np.ctypeslib.as_array(pointer, shape=(c.value * h.value * w.value,))
        if not np.isfinite(canvas[:: max(1, canvas.size // 4096)]).all():
            raise RuntimeError("the result holds values that are not finite")
        ph, pw, pc = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        pointer = library.unround_result_picture(result, ctypes.byref(ph), ctypes.byref(pw), ctypes.byref(pc))
        picture = np.ctypeslib.as_array(pointer, shape=(ph.value * pw.value * pc.value,))
        if not np.isfinite(picture[:: max(1, picture.size // 4096)]).all():
            raise RuntimeError("the picture holds values that are not finite")
        coefficients = 0
        for index in range(int(library.unround_result_components(result))):
            count = ctypes.c_uint64()
            library.unround_result_coefficients(result, index, ctypes.byref(count))
            coefficients += count.value
        # The planes are the canvas here (no cut); a one-channel picture is the planes.
        return canvas.nbytes + 8 * coefficients + (picture.nbytes if pc.value > 1 else 0)
    finally:
        library.unround_result_free(result)
        del kept


def _call_levels(image, out) -> int:
    """One solve through the C interface to 8-bit levels (unround_b200_solve_levels, blue-noise
    dither): levels in, the picture made and quantized on the device, its bytes out into `out`
    (host memory). Returns the bytes copied from the device."""
    import ctypes

    from unround import native

    library = native._library()
    settings = native._Settings(OPTIONS)
    given, kept = native._input_of(image)
    sizes = (ctypes.c_uint64 * 3)()
    message = ctypes.create_string_buffer(4096)
    status = library.unround_b200_solve_levels(ctypes.byref(given), settings.handle, 0, 1,
                                               out.ctypes.data_as(ctypes.c_void_p), out.nbytes, sizes, message, 4096)
    if status != 0:
        raise RuntimeError(message.value.decode())
    del kept
    return int(sizes[0] * sizes[1] * sizes[2])


MIX_ITERATIONS = 300


def _call_batch(images, options) -> int:
    """The batched solve through the C interface, as a C or cgo caller makes it:
    unround_b200_solve_batch on host arrays (levels in; every picture's binary64 canvas,
    coefficients and RGB picture out, into its result), then each result's canvas and picture
    read on the host. Returns the results' bytes copied from the device."""
    import ctypes

    import numpy as np

    from unround import native

    library = native._library()
    count = len(images)
    handles = [native._Settings(o) for o in options]
    inputs = (native._Input * count)()
    kept = []
    for n, image in enumerate(images):
        given, held = native._input_of(image)
        inputs[n] = given
        kept.append(held)
    settings = (ctypes.c_void_p * count)(*(h.handle for h in handles))
    results = (ctypes.c_void_p * count)()
    timing = native._BatchTiming()
    message = ctypes.create_string_buffer(4096)
    status = library.unround_b200_solve_batch(count, inputs, settings, results, ctypes.byref(timing), message, 4096)
    try:
        if status != 0:
            raise RuntimeError(message.value.decode())
        copied = 0
        for n in range(count):
            c, h, w = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
            pointer = library.unround_result_canvas(results[n], ctypes.byref(c), ctypes.byref(h), ctypes.byref(w))
            canvas = np.ctypeslib.as_array(pointer, shape=(c.value * h.value * w.value,))
            pointer = library.unround_result_picture(results[n], ctypes.byref(h), ctypes.byref(w), ctypes.byref(c))
            picture = np.ctypeslib.as_array(pointer, shape=(h.value * w.value * c.value,))
            if not (np.isfinite(canvas[:: max(1, canvas.size // 1024)]).all()
                    and np.isfinite(picture[:: max(1, picture.size // 1024)]).all()):
                raise RuntimeError("a result holds values that are not finite")
            coefficients = 0
            for index in range(int(library.unround_result_components(results[n]))):
                number = ctypes.c_uint64()
                library.unround_result_coefficients(results[n], index, ctypes.byref(number))
                coefficients += number.value
            # The canvas and coefficients; the planes where the canvas is larger than the picture;
            # the interleaved picture of more than one channel.
            planes = picture.nbytes if canvas.size != picture.size else 0
            copied += canvas.nbytes + 8 * coefficients + planes + (picture.nbytes if c.value > 1 else 0)
        return copied
    finally:
        for n in range(count):
            if results[n]:
                library.unround_result_free(results[n])
        del kept


# Algorithmic bytes per sample-iteration of a fused iteration: TV 3 fields, TGV 8, read and
# written in binary32, and the int16 levels (2 B a sample in grey, 1 B in 4:2:0).
def _picture_bytes(entry) -> float:
    samples = entry.image.height * entry.image.width * (3 if entry.colour else 1)
    fields = 8 if entry.method == "tgv" else 3
    return samples * (fields * 8.0 + (1.0 if entry.colour else 2.0))


def _mix_measure(pictures: int, warmup: int, seed: int) -> dict:
    """The batched solve of a seeded mix against the same pictures solved one after another."""
    from unround import native, synthetic

    mix = synthetic.mix(pictures, seed=seed, iterations=MIX_ITERATIONS)
    images, options = [e.image for e in mix], [e.options for e in mix]
    pixels = sum(e.image.height * e.image.width for e in mix)
    for _ in range(max(1, warmup)):
        native.solve_batch(images[:2], options[:2])  # warm the call path and the kernels
    with Clocks(0) as clocks:
        _, timing = native.solve_batch(images, options)
    # End to end through the C interface (the results' pinned blocks warmed by the call above).
    began = time.perf_counter()
    d2h = _call_batch(images, options)
    e2e_seconds = time.perf_counter() - began
    batched = pixels * timing.iterations / (timing.milliseconds / 1e3) / 1e6
    alone_ms = 0.0
    for image, option in zip(images, options):
        measured, _ = native.measure(image, option, warmup=0, iterations=timing.iterations)
        alone_ms += measured.milliseconds
    alone = pixels * timing.iterations / (alone_ms / 1e3) / 1e6
    peak, peak_kind = _peaks()
    moved = sum(_picture_bytes(e) for e in mix) * timing.iterations
    alone_gbs, batched_gbs = moved / (alone_ms / 1e3) / 1e9, moved / (timing.milliseconds / 1e3) / 1e9
    return {
        "mix": mix, "timing": timing, "pixels": pixels, "batched": batched, "alone": alone, "alone_ms": alone_ms,
        "e2e": pixels * MIX_ITERATIONS / e2e_seconds / 1e6, "d2h": d2h, "clocks": clocks.summary(),
        "h2d": sum(sum(c.coefficients.nbytes for c in e.image.components) for e in mix),
        # The image-at-a-time path's share of the peak bounds what batching can gain: at best
        # the whole mix moves its bytes at the peak.
        "roofline": {"algorithmic_bytes_per_iteration": moved / timing.iterations, "peak": peak,
                     "peak_kind": peak_kind, "image_at_a_time_gbs": alone_gbs,
                     "image_at_a_time_frac": alone_gbs / peak, "batched_gbs": batched_gbs,
                     "batched_frac": batched_gbs / peak, "speedup_ceiling": peak / alone_gbs},
    }


def _mix_arm(args: argparse.Namespace, rank: int, world: int) -> None:
    """The batched solve of a seeded mix of pictures (sides multiples of 16 in [256, 2048], grey
    or 4:2:0 colour, quality 10..90, TV or TGV, alpha log-uniform in [0.3, 3], 300 iterations)
    in one CUDA graph, against the same pictures solved one after another with plain launches.
    value: all pictures' pixel-iterations over the batched iterations' device time (CUDA events
    around the graph launch); image_at_a_time: the same over the sum of each picture's
    iteration loop alone (unround_b200_measure, CUDA events); e2e: through the C interface's
    batch call with host arrays (levels in, binary64 results out), wall clock. Each rank solves
    its own mix (weak scaling); rank 0 prints."""
    m = _mix_measure(args.pictures, args.warmup, 3 + rank)
    mix, timing = m["mix"], m["timing"]
    if rank != 0:
        return
    line = {
        "metric": f"batched TV/TGV mix Mpx*iter/s on 1 B200 ({args.pictures} pictures, {MIX_ITERATIONS} iterations)",
        "value": m["batched"], "unit": "Mpx*iter/s", "n_gpus": world, "steps": 1, "warmup": args.warmup,
        "ms_per_step": timing.milliseconds, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded mix: sides 16k in [256, 2048], grey/4:2:0, Q 10..90, TV/TGV)",
        "config": {"workload": f"mix-{args.pictures}", "pictures": args.pictures, "pixels": m["pixels"],
                   "samples": timing.samples, "iterations_timed": timing.iterations,
                   "tgv": sum(e.method == "tgv" for e in mix), "colour": sum(e.colour for e in mix),
                   "l2": "state larger than L2, no flush"},
        "image_at_a_time": {"value": m["alone"], "unit": "Mpx*iter/s", "ms": m["alone_ms"]},
        "speedup_vs_image_at_a_time": m["batched"] / m["alone"],
        "roofline": m["roofline"],
        "e2e": {"value": m["e2e"], "unit": "Mpx*iter/s", "h2d_bytes_per_step": m["h2d"], "d2h_bytes_per_step": m["d2h"]},
        "gpu_launches": timing.launches_per_iteration * timing.iterations,
        "clocks": m["clocks"],
    }
    print(json.dumps(line))


SAMPLES_BYTES = 18.0  # the samples' primal step: x, p1, p2 and the 16-bit level read, x~ written
SAMPLES_FUSED_BYTES = DUAL_BYTES + 6.0  # the fused sweep: the dual step's, the level read, x~ written


def _samples_arm(args: argparse.Namespace, rank: int, world: int) -> None:
    """Pictures of rounded samples (the PNG path, unround_b200_solve_samples): the bench's
    4032x3024 colour picture as 8-bit RGB levels, TGV (alpha1 1, alpha0 2), 500 iterations.
    value: the iteration loop's device time (unround_b200_measure_samples, CUDA events); e2e:
    the C call with host levels in and the binary64 result out; roofline: the dual sweep and
    the samples' primal step, each against its algorithmic bytes."""
    import ctypes

    import numpy as np

    from unround import native, synthetic
    from unround.sharding import max_over_ranks

    rgb = synthetic.colour(HEIGHT, WIDTH, quality=75, seed=rank, noise=3.0).samples
    levels = np.ascontiguousarray(np.clip(np.rint(rgb), 0, 255).astype(np.uint16))
    options = [*OPTIONS[:6], "--iterations", str(ITERATIONS), "--tolerance", "0", "--record-every", "0"]
    with Clocks(0) as clocks:
        timing = native.measure_samples(levels, 8, options, warmup=max(3, args.warmup) * 10,
                                        iterations=args.steps * ITERATIONS)
    # Beside: the loop as one launch an iteration, the primal step in the fused sweep of
    # iteration.cu (UNROUND_B200_KERNELS=fused) or in the dual sweep (=sweep).
    others = {}
    for mode in ("fused", "sweep"):
        os.environ["UNROUND_B200_KERNELS"] = mode
        try:
            others[mode] = native.measure_samples(levels, 8, options, warmup=30, iterations=ITERATIONS)
        finally:
            del os.environ["UNROUND_B200_KERNELS"]

    seconds = max_over_ranks(timing.milliseconds / 1e3)
    pixels = timing.pixels
    value = world * pixels * args.steps * ITERATIONS / seconds / 1e6
    library = native._library()
    settings = native._Settings(options)

    def call() -> int:
        result = ctypes.c_void_p()
        message = ctypes.create_string_buffer(4096)
        status = library.unround_b200_solve_samples(levels.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), HEIGHT,
                                                    WIDTH, 3, 8, settings.handle, native._OBSERVER(), None,
                                                    ctypes.byref(result), message, 4096)
        if status != 0:
            raise RuntimeError(message.value.decode())
        try:
            c, h, w = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
            pointer = library.unround_result_picture(result, ctypes.byref(h), ctypes.byref(w), ctypes.byref(c))
            picture = np.ctypeslib.as_array(pointer, shape=(h.value * w.value * c.value,))
            if not np.isfinite(picture[:: max(1, picture.size // 4096)]).all():
                raise RuntimeError("the result holds values that are not finite")
            return 2 * picture.nbytes  # the canvas and the interleaved picture
        finally:
            library.unround_result_free(result)

    call()  # warm the call path
    began = time.perf_counter()
    for _ in range(args.steps):
        d2h = call()
    e2e_seconds = max_over_ranks(time.perf_counter() - began)
    peak, peak_kind = _peaks()
    dual = DUAL_BYTES * timing.samples / (timing.dual_milliseconds / 1e3) / 1e9
    primal = SAMPLES_BYTES * timing.samples / (timing.primal_milliseconds / 1e3) / 1e9
    iteration = (DUAL_BYTES + SAMPLES_BYTES) * timing.samples / (seconds / (args.steps * ITERATIONS)) / 1e9
    if rank != 0:
        return
    line = {
        "metric": "TGV PDHG of rounded samples Mpx*iter/s on 1 B200 (4032x3024 RGB 8-bit, 500 iterations)",
        "value": value, "unit": "Mpx*iter/s",
        "msample_iter_per_s": world * timing.samples * args.steps * ITERATIONS / seconds / 1e6,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": seconds / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (the bench's colour picture, RGB, 8-bit levels)",
        "config": {"workload": "samples-rgb8-4032x3024", "iterations_per_step": ITERATIONS, "alpha1": 1.0,
                   "alpha0": 2.0, "samples": timing.samples, "l2": "state larger than L2, no flush"},
        "roofline": {"bound": "hbm", "kernel": "dual_kernel<tgv,3,coupled>", "achieved": dual, "peak": peak,
                     "unit": "GB/s", "frac": dual / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_sample": DUAL_BYTES, "dual_ms": timing.dual_milliseconds,
                     "samples_primal_achieved": primal, "samples_primal_frac": primal / peak,
                     "samples_primal_bytes_per_sample": SAMPLES_BYTES, "primal_ms": timing.primal_milliseconds,
                     "iteration_achieved": iteration, "iteration_frac": iteration / peak,
                     "one_launch": {mode: {"iteration_ms": t.milliseconds / t.iterations,
                                           "bytes_per_sample": SAMPLES_FUSED_BYTES,
                                           "achieved": SAMPLES_FUSED_BYTES * t.samples / (t.milliseconds / t.iterations)
                                           / 1e6}
                                    for mode, t in others.items()}},
        "e2e": {"value": world * pixels * args.steps * ITERATIONS / e2e_seconds / 1e6, "unit": "Mpx*iter/s",
                "h2d_bytes_per_step": int(levels.nbytes), "d2h_bytes_per_step": d2h},
        "gpu_launches": timing.launches_per_iteration * args.steps * ITERATIONS,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))


LARGE_OPTIONS = ["--method", "tgv", "--alpha1", "1.5", "--alpha0", "3", "--iterations", "1000", "--tolerance", "0",
                 "--record-every", "50"]


def _records_arm(args: argparse.Namespace, rank: int, world: int) -> None:
    """The bench workload through unround_solve with a record every 10 iterations, the
    reference's default (each record: the tilde point kept by the dual and primal steps, its
    norms, conjugates and data term summed on the device, one copy back), against the same solve
    recording at its last iteration only. value: Mpx*iter/s with the records; ms_per_record the
    difference over the records taken. Each rank solves its own picture; rank 0 prints."""
    from unround import native

    image = _workload(seed=rank)
    recording = [*OPTIONS[:-1], "10"]
    for _ in range(max(1, args.warmup)):
        _call(image)
    plain_s, recorded_s = [], []
    with Clocks(0) as clocks:
        for _ in range(max(1, args.steps)):
            began = time.perf_counter()
            _call(image)
            plain_s.append(time.perf_counter() - began)
            began = time.perf_counter()
            _call(image, recording)
            recorded_s.append(time.perf_counter() - began)
    records = ITERATIONS // 10 + 1
    pixels = HEIGHT * WIDTH
    if rank != 0:
        return
    value = pixels * ITERATIONS / min(recorded_s) / 1e6
    print(json.dumps({
        "metric": METRIC + ", a record every 10 iterations", "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": min(recorded_s) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (the bench workload)",
        "config": {"workload": "tgv-colour-4032x3024-420-records", "record_every": 10, "records": records,
                   "call": "unround_solve on host arrays"},
        "without_records": {"value": pixels * ITERATIONS / min(plain_s) / 1e6, "ms_per_step": min(plain_s) * 1e3},
        "ms_per_record": (min(recorded_s) - min(plain_s)) * 1e3 / (records - 1),
        "clocks": clocks.summary(),
    }))


TV_GREY_OPTIONS = ["--method", "tv", "--alpha", "1", "--iterations", "200", "--tolerance", "0", "--record-every", "0",
                   "--step-ratio", "1", "--step-product", "0.99", "--norm-squared", "7.92"]


def _tv_grey_arm(args: argparse.Namespace, rank: int, world: int) -> None:
    """The small TV solve: a 512 x 512 grey picture of the generator at quality 50, TV with
    alpha 1, 200 iterations, tau = sigma = sqrt(1/8) (step ratio 1, product 0.99, norm squared
    7.92). Its state (3 MB) lives in L2 and a launch is short, so the figure is absolute, not a
    fraction of HBM. value: the iteration loop's device time (CUDA events), K solves of 200
    iterations; e2e: the drop-in call with host arrays; cpu_baseline: the reference's solver on
    the host cores, one whole solve with every thread and with one, run first."""
    from unround import native, synthetic

    image = synthetic.grey(512, 512, quality=50, seed=1 + rank).image
    iterations = 200
    cpu = None
    if world == 1 and rank == 0:
        from oracle import reference

        if reference.available():
            components = [(c.coefficients, c.quant_table.reshape(64), c.h_samp_factor, c.v_samp_factor)
                          for c in image.components]
            cpu = {}
            for threads in (os.cpu_count() or 1, 1):
                best = None
                for _ in range(3):
                    began = time.perf_counter()
                    reference.solve(512, 512, 1, components, [*TV_GREY_OPTIONS, "--threads", str(threads)])
                    seconds = time.perf_counter() - began
                    best = seconds if best is None else min(best, seconds)
                cpu[threads] = 512 * 512 * iterations / best / 1e6
    with Clocks(0) as clocks:
        timing, _ = native.measure(image, TV_GREY_OPTIONS, warmup=max(3, args.warmup) * iterations,
                                   iterations=max(1, args.steps) * iterations)
    value = 512 * 512 * max(1, args.steps) * iterations / (timing.milliseconds / 1e3) / 1e6
    native.solve(image, TV_GREY_OPTIONS)  # warm the call path
    began = time.perf_counter()
    for _ in range(max(1, args.steps)):
        native.solve(image, TV_GREY_OPTIONS)
    e2e_seconds = (time.perf_counter() - began) / max(1, args.steps)
    if rank != 0:
        return
    line = {
        "metric": "TV PDHG Mpx*iter/s on 1 B200 (512x512 grey, quality 50, 200 iterations)", "value": value,
        "unit": "Mpx*iter/s", "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
        "ms_per_step": timing.milliseconds / max(1, args.steps), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded piecewise-smooth, quality 50)",
        "config": {"workload": "tv-grey-512", "iterations": iterations, "tau_sigma": "sqrt(1/8)",
                   "l2": "state 3 MB: L2-resident, absolute figure"},
        "e2e": {"value": 512 * 512 * iterations / e2e_seconds / 1e6, "unit": "Mpx*iter/s",
                "h2d_bytes_per_step": int(image.components[0].coefficients.nbytes), "d2h_bytes_per_step": None,
                "call": "unround.native.solve (the drop-in, with the model's arrays made and copied)"},
        "gpu_launches": timing.launches_per_iteration * iterations * max(1, args.steps),
        "clocks": clocks.summary(),
    }
    if cpu:
        threads = os.cpu_count() or 1
        line["cpu_baseline"] = {"value": cpu[threads], "unit": "Mpx*iter/s", "cores": threads, "kind": "reference",
                                "sample": "one whole solve (200 iterations with its set-up), best of 3",
                                "one_thread": {"value": cpu[1], "cores": 1}}
    print(json.dumps(line))


def _large_arm(args: argparse.Namespace, rank: int, world: int) -> None:
    """The large single solve: 8192^2 TGV (alpha0 3, alpha1 1.5), 1000 iterations (--side: a
    smaller square of the same generator and table, for a capture of its kernels). value:
    the iteration loop's device time (CUDA events, no records); e2e: the drop-in solve with the
    primal-dual gap recorded every 50 iterations, host arrays in and out; and the binary64 check
    that every coefficient of all 1,048,576 blocks lies in its interval."""
    import numpy as np

    from unround import native, synthetic

    made = synthetic.large(args.side, seed=5 + rank)
    image = made.image
    iterations = 1000
    timed_options = [*LARGE_OPTIONS[:-2], "--record-every", "0"]
    with Clocks(0) as clocks:
        timing, _ = native.measure(image, timed_options, warmup=max(3, args.warmup) * 10, iterations=iterations)
    pixels = timing.pixels
    value = pixels * iterations / (timing.milliseconds / 1e3) / 1e6
    began = time.perf_counter()
    decoded = native.solve(image, LARGE_OPTIONS)
    e2e_seconds = time.perf_counter() - began
    lower = native.model(image, LARGE_OPTIONS, 0, 0)
    upper = native.model(image, LARGE_OPTIONS, 0, 1)
    zeta = decoded.coefficients[0].reshape(-1)
    inside = bool(np.all((zeta >= lower) & (zeta <= upper)))
    history = decoded.result.history
    peak, peak_kind = _peaks()
    if rank != 0:
        return
    line = {
        "metric": f"TGV PDHG Mpx*iter/s on 1 B200 ({args.side}x{args.side} grey, custom table, 1000 iterations)",
        "value": value, "unit": "Mpx*iter/s", "n_gpus": world, "steps": 1, "warmup": max(3, args.warmup) * 10,
        "ms_per_step": timing.milliseconds, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded piecewise-smooth + noise sigma 2, table steps U{1..64})",
        "config": {"workload": f"tgv-grey-{args.side}-custom", "alpha1": 1.5, "alpha0": 3.0, "iterations": iterations,
                   "samples": timing.samples, "l2": f"state {17 * 4 * timing.samples / 1e9:.2f} GB"},
        "roofline": {"bound": "hbm", "kernel": "dual_tma_kernel<tgv,1>", "achieved":
                     DUAL_BYTES * timing.samples / (timing.dual_milliseconds / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "peak_kind": peak_kind,
                     "frac": DUAL_BYTES * timing.samples / (timing.dual_milliseconds / 1e3) / 1e9 / peak,
                     "iteration_bytes_per_sample": 66.0,
                     "iteration_frac": 66.0 * timing.samples / (timing.milliseconds / iterations / 1e3) / 1e9 / peak,
                     "dual_ms": timing.dual_milliseconds, "primal_ms": timing.primal_milliseconds},
        "gap_per_sample_every_50": [float(g) / timing.samples for g in history.gap],
        "record_iterations": [int(n) for n in history.iterations],
        "all_blocks_inside_intervals_fp64": inside, "blocks": int(zeta.size // 64),
        "e2e": {"value": pixels * iterations / e2e_seconds / 1e6, "unit": "Mpx*iter/s",
                "h2d_bytes_per_step": int(image.components[0].coefficients.nbytes),
                "d2h_bytes_per_step": int(decoded.canvas.nbytes + zeta.nbytes)},
        "gpu_launches": timing.launches_per_iteration * iterations,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))


def _unrolled_forward_launches(iterations: int) -> int:
    """The start, N primal steps and N - 1 dual steps."""
    return 2 * iterations


def _unrolled_backward_launches(iterations: int, every: int) -> int:
    """Per segment of checkpoints K apart: the recomputed dual steps and primal steps, then the
    dual steps' adjoints (N - 1) and the primal steps' adjoints (N)."""
    launches = 0
    for k0 in range(0, iterations, every):
        k1 = min(k0 + every, iterations)
        launches += (k1 - k0 - 1) + max(k1 - k0 - 2, 0) + (1 if k1 - k0 > 1 and k1 < iterations else 0)
    return launches + (iterations - 1) + iterations


def _unrolled_measure(steps: int, warmup: int, rank: int) -> dict:
    """The differentiable unrolled TGV solve of 16 greyscale 512x512 pictures (quality 30), 100
    iterations: per step one forward pass with the loss (MSE against the clean pictures), one
    forward and backward pass (the adjoint) to the gradients of every picture's alpha0, alpha1, tau
    and sigma with checkpoints every 10 iterations, and the same with a checkpoint every iteration
    (no state recomputed; 9 planes an iteration in HBM); device times by CUDA events."""
    import numpy as np
    import torch

    from unround import synthetic
    from unround.unrolled import UnrolledProblem, unrolled_tgv

    pictures, side, iterations, every = 16, 512, 100, 10
    made = [synthetic.grey(side, side, quality=30, seed=100 * rank + s, noise=2) for s in range(pictures)]
    options = ["--method", "tgv", "--alpha1", "1", "--alpha0", "2"]
    problem = UnrolledProblem([m.image for m in made], options, iterations=iterations, checkpoint_every=every)
    clean = torch.tensor(np.stack([m.samples for m in made]), dtype=torch.float32, device="cuda")
    base = [torch.full((pictures,), v, dtype=torch.float32, device="cuda")
            for v in (2.0, 1.0, problem.tau, problem.sigma)]

    def forward_only():
        with torch.no_grad():
            out = unrolled_tgv(problem, *base)
            return torch.mean((out - clean) ** 2)

    def forward_backward():
        leaves = [b.clone().requires_grad_(True) for b in base]
        loss = torch.mean((unrolled_tgv(problem, *leaves) - clean) ** 2)
        loss.backward()
        return leaves

    kept = UnrolledProblem([m.image for m in made], options, iterations=iterations, checkpoint_every=1)

    def forward_backward_kept():
        leaves = [b.clone().requires_grad_(True) for b in base]
        torch.mean((unrolled_tgv(kept, *leaves) - clean) ** 2).backward()

    for _ in range(max(3, warmup)):
        forward_only()
        forward_backward()
        forward_backward_kept()
    torch.cuda.synchronize()
    start, mid, end, last = (torch.cuda.Event(enable_timing=True) for _ in range(4))
    steps = max(1, steps)
    with Clocks(0) as clocks:
        start.record()
        for _ in range(steps):
            forward_only()
        mid.record()
        for _ in range(steps):
            leaves = forward_backward()
        end.record()
        for _ in range(steps):
            forward_backward_kept()
        last.record()
        torch.cuda.synchronize()
    grads = torch.stack([leaf.grad for leaf in leaves]).cpu()  # the step's result read on the host
    # End to end: levels in from the host (the problem made from the files' levels), gradients out.
    began = time.perf_counter()
    problem_e2e = UnrolledProblem([m.image for m in made], options, iterations=iterations, checkpoint_every=every)
    leaves = [b.clone().requires_grad_(True) for b in base]
    torch.mean((unrolled_tgv(problem_e2e, *leaves) - clean) ** 2).backward()
    e2e_grads = torch.stack([leaf.grad for leaf in leaves]).cpu()
    return {"pictures": pictures, "side": side, "iterations": iterations, "every": every, "steps": steps,
            "forward_ms": start.elapsed_time(mid) / steps, "both_ms": mid.elapsed_time(end) / steps,
            "kept_ms": end.elapsed_time(last) / steps, "kept_bytes": kept.checkpoint_floats * 4,
            "grad_finite": bool(torch.isfinite(grads).all()) and bool(torch.isfinite(e2e_grads).all()),
            "e2e_seconds": time.perf_counter() - began, "e2e_d2h": int(e2e_grads.numel() * 4),
            "h2d": sum(m.image.components[0].coefficients.nbytes for m in made), "clocks": clocks.summary()}


def _unrolled_arm(args: argparse.Namespace, rank: int, world: int) -> None:
    """The unrolled solve's line (_unrolled_measure). value: pixel-iterations of the forward and
    backward pass per second; forward: the same of the forward pass alone; ratio: (forward +
    backward) / forward; every_iterate_kept: the same with a checkpoint every iteration."""
    m = _unrolled_measure(args.steps, args.warmup, rank)
    if rank != 0:
        return
    pixels, iterations, every, steps = m["pictures"] * m["side"] ** 2, m["iterations"], m["every"], m["steps"]
    line = {
        "metric": "unrolled TGV forward+adjoint Mpx*iter/s on 1 B200 (16 x 512x512, 100 iterations, checkpoints 10)",
        "value": pixels * iterations / (m["both_ms"] / 1e3) / 1e6, "unit": "Mpx*iter/s", "n_gpus": world,
        "steps": steps, "warmup": max(3, args.warmup), "ms_per_step": m["both_ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded piecewise-smooth + noise sigma 2, quality 30)",
        "config": {"workload": "unrolled-tgv-16x512", "pictures": m["pictures"], "iterations": iterations,
                   "checkpoint_every": every, "loss": "MSE against the clean pictures",
                   "l2": "state 16 x 512^2 x 9 fields = 151 MB, larger than L2"},
        "forward": {"value": pixels * iterations / (m["forward_ms"] / 1e3) / 1e6, "ms": m["forward_ms"]},
        "forward_backward_over_forward": m["both_ms"] / m["forward_ms"],
        "backward_over_forward": (m["both_ms"] - m["forward_ms"]) / m["forward_ms"],
        "every_iterate_kept": {"checkpoint_every": 1, "ms": m["kept_ms"],
                               "forward_backward_over_forward": m["kept_ms"] / m["forward_ms"],
                               "checkpoint_bytes": m["kept_bytes"]},
        "grad_finite": m["grad_finite"],
        "e2e": {"value": pixels * iterations / m["e2e_seconds"] / 1e6, "unit": "Mpx*iter/s",
                "h2d_bytes_per_step": m["h2d"], "d2h_bytes_per_step": m["e2e_d2h"]},
        "gpu_launches": steps * (2 * _unrolled_forward_launches(iterations) + _unrolled_backward_launches(iterations, every)
                                 + _unrolled_forward_launches(iterations) + _unrolled_backward_launches(iterations, 1)),
        "clocks": m["clocks"],
    }
    print(json.dumps(line))


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=3)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", default="b200", choices=["b200", "reference"])
    parser.add_argument("--height", type=int, default=HEIGHT, help="a smaller picture for profiling")
    parser.add_argument("--width", type=int, default=WIDTH)
    parser.add_argument("--workload", default="tgv-colour",
                        choices=["tgv-colour", "mix", "unrolled", "large", "samples", "records", "tv-grey"],
                        help="mix: the batched solve of 64 uneven pictures against image-at-a-time launches; "
                             "unrolled: the differentiable unrolled TGV solve, forward and forward+adjoint")
    parser.add_argument("--pictures", type=int, default=64, help="pictures of the mix")
    parser.add_argument("--side", type=int, default=8192, help="side of the large workload's square picture")
    parser.add_argument("--mix-iterations", type=int, default=MIX_ITERATIONS,
                        help="iterations of each picture of the mix (fewer for a launch list)")
    args = parser.parse_args()
    globals()["HEIGHT"], globals()["WIDTH"] = args.height, args.width
    rank, local_rank, world = _rank()
    if world > 1:
        # One GPU per rank, made the process's only visible device before any CUDA call.
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local_rank)
    for path in (ROOT / "jpeg-unround_b200", ROOT):
        sys.path.insert(0, str(path))
    globals()["MIX_ITERATIONS"] = args.mix_iterations
    if args.workload == "mix":
        _mix_arm(args, rank, world)
        return
    if args.workload == "records":
        _records_arm(args, rank, world)
        return
    if args.workload == "tv-grey":
        _tv_grey_arm(args, rank, world)
        return
    if args.workload == "unrolled":
        _unrolled_arm(args, rank, world)
        return
    if args.workload == "large":
        _large_arm(args, rank, world)
        return
    if args.workload == "samples":
        _samples_arm(args, rank, world)
        return
    group = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        group = dist
    if args.impl == "reference":
        _reference_arm(args, rank)
        if group is not None:
            group.destroy_process_group()
        return

    import numpy as np

    from unround import native

    image = _workload(seed=rank)
    # The CPU baseline first, before any GPU work in this process (rank 0, one GPU only).
    cpu_baseline, theirs = _cpu_baseline(image) if (world == 1 and rank == 0) else (None, None)
    # Warm-up steps and timed steps of the device-resident loop.
    if group is not None:
        group.barrier()
    with Clocks(local_rank if world == 1 else 0) as clocks:
        timing, _ = native.measure(image, OPTIONS, warmup=args.warmup * ITERATIONS, iterations=args.steps * ITERATIONS)
    from unround.sharding import max_over_ranks

    seconds = max_over_ranks(timing.milliseconds / 1e3)  # the slowest rank's
    pixels = timing.pixels
    value = world * pixels * args.steps * ITERATIONS / seconds / 1e6
    # End to end through the drop-in call, host arrays in and out.
    if group is not None:
        group.barrier()
    levels_bytes = sum(c.coefficients.nbytes for c in image.components)
    _call(image)  # warm the call path
    began = time.perf_counter()
    for _ in range(args.steps):
        d2h = _call(image)
    e2e_seconds = max_over_ranks(time.perf_counter() - began)
    e2e = world * pixels * args.steps * ITERATIONS / e2e_seconds / 1e6
    # The same to 8-bit levels: only the quantized picture comes back.
    levels = np.empty(pixels * 3, dtype=np.uint8)
    _call_levels(image, levels)  # warm the call path
    began = time.perf_counter()
    for _ in range(args.steps):
        levels_d2h = _call_levels(image, levels)
    levels_seconds = max_over_ranks(time.perf_counter() - began)
    e2e_levels = world * pixels * args.steps * ITERATIONS / levels_seconds / 1e6
    # From a JPEG file's bytes: the host reads the coefficients, the rest as e2e.
    jpeg = _jpeg_file(seed=rank)
    _call_file(jpeg)  # warm the call path
    began = time.perf_counter()
    for _ in range(args.steps):
        file_d2h = _call_file(jpeg)
    file_seconds = max_over_ranks(time.perf_counter() - began)
    e2e_file = world * pixels * args.steps * ITERATIONS / file_seconds / 1e6
    # The records' cost at the reference's default (a record every 10 iterations, each with its
    # host round trip): solves through the drop-in call with and without them.
    recording = [*OPTIONS[:-1], "10"]
    native.solve(image, recording)
    plain_s, recorded_s = [], []
    for _ in range(2):
        began = time.perf_counter()
        native.solve(image, OPTIONS)
        plain_s.append(time.perf_counter() - began)
        began = time.perf_counter()
        recorded = native.solve(image, recording)
        recorded_s.append(time.perf_counter() - began)
    python_seconds = max_over_ranks(min(plain_s))  # every rank takes part, as in e2e
    record_count = len(recorded.result.history.iterations)
    records = {"record_every": 10, "records": record_count, "solve_ms": min(recorded_s) * 1e3,
               "solve_ms_without": min(plain_s) * 1e3,
               "ms_per_record": (min(recorded_s) - min(plain_s)) * 1e3 / max(record_count - 1, 1),
               "value": pixels * ITERATIONS / min(recorded_s) / 1e6, "unit": UNIT}
    parity = _parity(native.solve(image, OPTIONS), theirs, image) if theirs is not None else None
    # The batched mix beside (the batching workload): batched against image at a time.
    mixed = _mix_measure(64, 1, 3) if world == 1 else None
    # The unrolled solve beside (the differentiation workload): forward+backward against forward.
    unrolled = _unrolled_measure(3, 3, 0) if world == 1 else None
    peak, peak_kind = _peaks()
    copy = _copy_gbs()
    samples = timing.samples
    dual_achieved = DUAL_BYTES * samples / (timing.dual_milliseconds / 1e3) / 1e9
    iteration_seconds = seconds / (args.steps * ITERATIONS)
    iteration_achieved = ALGORITHMIC_BYTES * samples / iteration_seconds / 1e9
    traffic = _traffic()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT,
            "msample_iter_per_s": world * timing.samples * args.steps * ITERATIONS / seconds / 1e6,
            "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": seconds / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded piecewise-smooth per RGB channel + noise sigma 3, quality 75)",
            "config": {"workload": "tgv-colour-4032x3024-420", "iterations_per_step": ITERATIONS,
                       "alpha1": 1.0, "alpha0": 2.0, "samples": samples, "pixels": pixels,
                       "l2": "state larger than L2 (~3 GB), no flush", "parallelism": f"{world} independent images"},
            "roofline": {"bound": "hbm", "kernel": "dual_kernel<tgv,3,coupled>", "achieved": dual_achieved,
                         "peak": peak, "unit": "GB/s", "frac": dual_achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "algorithmic_bytes_per_sample": DUAL_BYTES,
                         "iteration_achieved": iteration_achieved, "iteration_frac": iteration_achieved / peak,
                         "iteration_bytes_per_sample": ALGORITHMIC_BYTES,
                         "dual_ms": timing.dual_milliseconds, "primal_ms": timing.primal_milliseconds,
                         "copy_gbs_this_box": copy, "frac_of_copy_this_box": dual_achieved / copy,
                         "iteration_frac_of_copy_this_box": iteration_achieved / copy},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": levels_bytes, "d2h_bytes_per_step": d2h},
            "e2e_levels": {"value": e2e_levels, "unit": UNIT, "h2d_bytes_per_step": levels_bytes,
                           "d2h_bytes_per_step": levels_d2h,
                           "call": "unround_b200_solve_levels, 8 bits, blue-noise dither"},
            "e2e_file": {"value": e2e_file, "unit": UNIT, "h2d_bytes_per_step": len(jpeg),
                         "d2h_bytes_per_step": file_d2h,
                         "call": "unround_decode of a JPEG file (quality 75, 4:2:0, Pillow-written) of the "
                                 "workload's picture; coefficients read on the host"},
            "e2e_python": {"value": world * pixels * ITERATIONS / python_seconds / 1e6, "unit": UNIT,
                           "call": "unround.native.solve, the Python drop-in: the result's arrays and the "
                                   "model's copied into NumPy (best of 2)"},
            "gpu_launches": timing.launches_per_iteration * args.steps * ITERATIONS,
            "clocks": clocks.summary(),
            "records": records,
        }
        if world == 1:
            line["cpu_baseline"] = cpu_baseline
            line["parity"] = parity
            line["mix"] = {"pictures": 64, "iterations_timed": mixed["timing"].iterations,
                           "batched": mixed["batched"], "image_at_a_time": mixed["alone"],
                           "speedup_vs_image_at_a_time": mixed["batched"] / mixed["alone"],
                           "roofline": mixed["roofline"], "e2e": mixed["e2e"], "unit": UNIT}
            line["unrolled"] = {"workload": "unrolled-tgv-16x512, 100 iterations", "forward_ms": unrolled["forward_ms"],
                                "forward_backward_ms": unrolled["both_ms"], "checkpoint_every": unrolled["every"],
                                "forward_backward_over_forward": unrolled["both_ms"] / unrolled["forward_ms"],
                                "backward_over_forward": (unrolled["both_ms"] - unrolled["forward_ms"])
                                                         / unrolled["forward_ms"],
                                "every_iterate_kept_over_forward": unrolled["kept_ms"] / unrolled["forward_ms"],
                                "every_iterate_kept_checkpoint_bytes": unrolled["kept_bytes"],
                                "grad_finite": unrolled["grad_finite"]}
        print(json.dumps(line))
    if group is not None:
        group.destroy_process_group()
    del np


if __name__ == "__main__":
    main()
