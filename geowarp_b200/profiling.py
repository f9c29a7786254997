"""Kernel timing through the library's CUDA-event instrumentation."""
import contextlib
import ctypes as C

from . import _lib as L


@contextlib.contextmanager
def kernel_timer():
    lib = L.load()
    lib.gw_profile_reset()
    lib.gw_profile_enable(1)
    rec = {}
    try:
        yield rec
    finally:
        lib.gw_profile_enable(0)
        for c in range(lib.gw_profile_count()):
            ms, n, b = C.c_double(0), C.c_int64(0), C.c_double(0)
            L.check(lib.gw_profile_read(c, C.byref(ms), C.byref(n), C.byref(b)), "gw_profile_read")
            rec[lib.gw_profile_name(c).decode()] = dict(ms=ms.value, launches=n.value, bytes=b.value)
        lib.gw_profile_reset()


def roofline_summary(rec, peaks, peak_kind="measured"):
    """Roofline entry for the kernel class with the largest total time."""
    tot = sum(v["ms"] for v in rec.values()) or 1.0
    name, v = max(rec.items(), key=lambda kv: kv[1]["ms"])
    peak = float(peaks.get("hbm_gbs", 6650.0))
    avg_ms = v["ms"] / max(v["launches"], 1)
    bytes_per_launch = v["bytes"] / max(v["launches"], 1)
    achieved = bytes_per_launch / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else 0.0
    return {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured" else "fallback 6.65 TB/s",
            "traffic": None, "launches": v["launches"], "avg_launch_us": avg_ms * 1e3,
            "bytes_per_launch": bytes_per_launch,
            "share_of_instrumented_time": v["ms"] / tot,
            "breakdown_ms": {k: round(x["ms"], 3) for k, x in rec.items()},
            "per_class": {k: _class_entry(x, peak) for k, x in rec.items() if x["launches"] > 0}}


def _class_entry(v, peak):
    """Average launch of one timing class: achieved algorithmic GB/s and its
    fraction of the HBM peak."""
    avg_ms = v["ms"] / max(v["launches"], 1)
    bpl = v["bytes"] / max(v["launches"], 1)
    gbs = bpl / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else 0.0
    return {"launches": v["launches"], "avg_launch_us": round(avg_ms * 1e3, 3), "bytes_per_launch": round(bpl),
            "achieved_gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
