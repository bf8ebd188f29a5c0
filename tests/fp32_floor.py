"""The accuracy floor of an FP32-state split-operator propagation, per packet.

Each packet is propagated in FP64 (numpy's FFT, the unitary Strang step of
spofft.f:120-191 without the reference's defects) twice: exactly, and with
the state rounded to FP32 once per step and nothing else.  The largest
|dC(t)| between the two over the run is the error a perfect FP32-state form
would have; a real FP32 kernel also rounds inside each FFT stage and phase,
so its error is a small multiple of this floor."""
import numpy as np


def fp32_state_floor(npts, sh, sm, vpot, psi, off, dt_au, nsteps):
    """max_t |dC(t)| of each packet (arrays concatenated over packets)."""
    out = []
    for k in range(len(npts)):
        n = int(npts[k])
        a, b = off[k], off[k + 1]
        kk = np.fft.fftfreq(n) * n
        T = (2 * np.pi * kk / (n * sh[k])) ** 2 / (2 * sm[k])
        h = np.exp(-0.5j * vpot[a:b] * dt_au)
        K = np.exp(-1j * T * dt_au)
        psi0 = np.asarray(psi[a:b], dtype=np.complex128)
        x = psi0.copy()
        y = psi0.copy()
        err = 0.0
        for _ in range(nsteps):
            x = h * np.fft.ifft(K * np.fft.fft(h * x))
            y = h * np.fft.ifft(K * np.fft.fft(h * y))
            y = y.astype(np.complex64).astype(np.complex128)
            err = max(err, abs(np.vdot(psi0, x) - np.vdot(psi0, y)))
        out.append(err)
    return np.asarray(out)
