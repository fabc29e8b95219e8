"""IR post-processing: the Chebyshev-I anti-alias design and the cascade
against the reference's own code compiled from its sources (oracle/_ref,
where it was built), the library's design against the oracle's, and the
pipeline's known answers.  The GPU pipeline itself is checked in
test_postprocess_gpu.py."""
import numpy as np
import pytest

import oracle
from virs_b200 import capi

SPECS = [(65856.0, 20000.0, 24000.0, 0.5, 90.0), (305500.0, 20000.0, 24000.0, 0.5, 90.0),
         (48000.0, 15000.0, 16000.0, 0.5, 90.0), (96000.0, 20000.0, 0.0, 1.0, 80.0), (44100.0, 5000.0, 9000.0, 0.1, 60.0)]


def _random_specs(n, seed=1):
    rng = np.random.default_rng(seed)
    out = list(SPECS)
    for _ in range(n):
        fs = float(rng.uniform(20000, 400000))
        fc = float(rng.uniform(0.05, 0.45) * fs)
        fst = float(fc * rng.uniform(1.05, 1.5)) if rng.random() < 0.8 else 0.0
        out.append((fs, fc, fst, float(rng.uniform(0.05, 2.0)), float(rng.uniform(30, 120))))
    return out


def test_oracle_design_and_cascade_match_the_reference_build():
    ref = oracle.ref_dsp()
    if ref is None:
        pytest.skip("reference filter code not built (oracle/Makefile target ref)")
    for s in _random_specs(300):
        want = np.zeros((64, 6))
        n = ref.ref_cheby_design(*s, want.ctypes.data, 64)
        got = oracle.cheby_design(*s)
        assert got.shape[0] == n and np.array_equal(got.view(np.uint64), want[:n].view(np.uint64)), s
    rng = np.random.default_rng(2)
    x = (rng.standard_normal(6000) * np.exp(-np.arange(6000) / 900.0)).astype(np.float32)
    for s in SPECS:
        sos = oracle.cheby_design(*s)
        want = np.zeros_like(x)
        ref.ref_cheby_process(sos.ctypes.data, sos.shape[0], x.ctypes.data, want.ctypes.data, x.size)
        assert np.array_equal(oracle.sos_df2t(sos, x).view(np.uint32), want.view(np.uint32))


def test_library_design_matches_the_oracle():
    for s in _random_specs(300, seed=3):
        assert np.array_equal(capi.design_chebyshev_lowpass(*s).view(np.uint64), oracle.cheby_design(*s).view(np.uint64)), s


def test_design_rejects_invalid_specs():
    for bad in [(48000.0, 30000.0, 0.0, 0.5, 90.0), (48000.0, 10000.0, 9000.0, 0.5, 90.0), (0.0, 1.0, 0.0, 0.5, 90.0)]:
        with pytest.raises(capi.VirsError) as e:
            capi.design_chebyshev_lowpass(*bad)
        assert e.value.status == capi.E_ARG


def test_design_is_a_chebyshev_lowpass():
    """Unit DC gain, ripple within the spec in the passband, attenuation at
    the stop edge."""
    fs, fc, fst = 65856.0, 20000.0, 24000.0
    sos = oracle.cheby_design(fs, fc, fst, 0.5, 90.0)

    def mag_db(f):
        z = np.exp(1j * 2 * np.pi * f / fs)
        h = np.prod([(b0 + b1 / z + b2 / z ** 2) / (a0 + a1 / z + a2 / z ** 2) for b0, b1, b2, a0, a1, a2 in sos])
        return 20 * np.log10(abs(h))

    assert abs(mag_db(0.0)) < 1e-9
    assert all(-0.5 - 1e-6 <= mag_db(f) <= 1e-6 for f in np.linspace(10.0, fc, 400)) or \
        all(-1e-6 <= mag_db(f) <= 0.5 + 1e-6 for f in np.linspace(10.0, fc, 400))
    assert mag_db(fst) <= -90.0 + 0.5


def test_resampling_keeps_a_passband_tone():
    """A 1 kHz tone at the simulation rate comes out at 48 kHz with the same
    frequency and, after normalisation, unit peak."""
    dt = np.float32(1.0 / 65856.0)
    steps = 6586
    t = np.arange(steps, dtype=np.float64) * float(dt)
    x = np.sin(2 * np.pi * 1000.0 * t).astype(np.float32)[None, :]
    sos = oracle.cheby_design(float(np.float32(1.0) / dt), 20000.0, 24000.0)
    y = oracle.postprocess(x, float(dt), 48000.0, sos, normalize=True)[0]
    assert y.size == int(48000.0 * (steps * float(dt)))
    assert abs(np.abs(y).max() - 1.0) < 1e-6
    seg = y[2000:]
    spec = np.abs(np.fft.rfft(seg * np.hanning(seg.size)))
    f = np.fft.rfftfreq(seg.size, 1.0 / 48000.0)
    assert abs(f[np.argmax(spec)] - 1000.0) < 48000.0 / seg.size * 1.5


def _tone_response(resample, fs, rate, f, n=24000):
    """Amplitude of the output component at f (least squares over the middle
    half) and the output's whole RMS amplitude, for a unit sine at f."""
    t = np.arange(n) / fs
    y = resample(np.sin(2 * np.pi * f * t).astype(np.float32)).astype(np.float64)
    tt = np.arange(y.size) / rate
    sl = slice(y.size // 4, 3 * y.size // 4)
    A = np.stack([np.sin(2 * np.pi * f * tt[sl]), np.cos(2 * np.pi * f * tt[sl])], 1)
    c, *_ = np.linalg.lstsq(A, y[sl], rcond=None)
    return float(np.hypot(*c)), float(np.sqrt(2.0 * np.mean(y[sl] ** 2)))


def test_resampling_chains_passband_and_stopband():
    """The two resampling chains of the library at the reference's default
    simulation rate (cell 343 / 88200 m, fs = 305.5 kHz) to 48 kHz, as
    measured on tones: the Chebyshev-I cascade (0.45 / 0.5 x 48 kHz edges,
    0.5 dB ripple, 90 dB, 13 sections) with linear interpolation ripples by
    up to 0.43 dB in 100 Hz - 20 kHz and leaks at most -102 dB from 24.5 to
    140 kHz; the Kaiser-windowed sinc (245 half-taps, beta 10.06, cutoff
    0.9167) is flat to 0.001 dB and leaks at most -111 dB.  kfr's
    resample_quality::high, which the reference uses, is absent, so neither
    is pinned to it; these are the figures the two chains are held to."""
    h = np.float32(343.0 / (22050 * 2 * 2))
    fs = float(oracle.filter_fs(h))
    rate = 48000.0
    n = 24000
    m = int(rate * n / fs)
    sos = oracle.cheby_design(fs, 0.45 * rate, 0.5 * rate, 0.5, 90.0)
    sim_rate = float(np.float32(1.0) / np.float32(1.0 / fs))

    def linear(x):
        out = np.zeros(m, np.float32)
        y = np.ascontiguousarray(oracle.sos_df2t(sos, x))
        oracle.lib().vo_resample(y.ctypes.data_as(oracle.C.c_void_p), oracle.C.c_uint64(n), oracle.C.c_double(sim_rate),
                                 oracle.C.c_double(rate), out.ctypes.data_as(oracle.C.c_void_p), oracle.C.c_uint64(m),
                                 oracle.C.c_int(0))
        return out

    def sinc(x):
        return oracle.resample_sinc(x, fs, rate, m, 245, 10.06, 0.9167)

    passband = [100.0, 1000.0, 3000.0, 5000.0, 10000.0, 15000.0, 18000.0, 20000.0]
    stopband = [24500.0, 26000.0, 30000.0, 40000.0, 60000.0, 100000.0, 140000.0]
    lin_pb = max(abs(20 * np.log10(_tone_response(linear, fs, rate, f, n)[0])) for f in passband)
    lin_sb = max(20 * np.log10(_tone_response(linear, fs, rate, f, n)[1]) for f in stopband)
    snc_pb = max(abs(20 * np.log10(_tone_response(sinc, fs, rate, f, n)[0])) for f in passband)
    snc_sb = max(20 * np.log10(_tone_response(sinc, fs, rate, f, n)[1]) for f in stopband)
    print(f"linear chain: ripple {lin_pb:.3f} dB, stop {lin_sb:.1f} dB; sinc: ripple {snc_pb:.4f} dB, stop {snc_sb:.1f} dB")
    assert lin_pb <= 0.5 and lin_sb <= -100.0
    assert snc_pb <= 0.001 and snc_sb <= -110.0
