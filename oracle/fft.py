"""3/2-dealiased real FFTs, NumPy FP64 (oracle; test infrastructure only).

Restates ``src/dnsjax/fft.py`` and the transform wrappers of
``src/dnsjax/operators.py``.  ``norm="forward"`` everywhere: the forward
transform divides by N, the inverse applies no factor.  Nyquist modes are
never stored.  ``numpy.fft`` implements the same transform definitions as
``jax.numpy.fft`` (the reference's FFT dependency, jax 0.10.0 per
``uv.lock:42-58``).  With oracle.parallel threads, each transform's lines
are split over them (bitwise the same result).
"""

from __future__ import annotations

import numpy as np

from . import parallel

NORM = "forward"


def zeropad_fft(a: np.ndarray, n: int, axis: int) -> np.ndarray:
    """fft.py:41-88: insert zeros between positive and negative modes."""
    N = a.shape[axis] + 1
    if n < N or (n - N) % 2:
        raise ValueError("bad zero-pad size")
    shape = list(a.shape)
    shape[axis] = n
    out = np.zeros(shape, dtype=a.dtype)
    src = [slice(None)] * a.ndim
    dst = [slice(None)] * a.ndim
    src[axis] = slice(None, N // 2)
    dst[axis] = slice(None, N // 2)
    out[tuple(dst)] = a[tuple(src)]
    src[axis] = slice(N // 2, None)
    dst[axis] = slice(n - N // 2 + 1, None)
    out[tuple(dst)] = a[tuple(src)]
    return out


def truncate_fft(a: np.ndarray, n: int, axis: int) -> np.ndarray:
    """fft.py:91-137: keep n/2 positive and n/2-1 negative modes."""
    N = a.shape[axis]
    if n > N or (N - n) % 2:
        raise ValueError("bad truncation size")
    shape = list(a.shape)
    shape[axis] = n - 1
    out = np.zeros(shape, dtype=a.dtype)
    src = [slice(None)] * a.ndim
    dst = [slice(None)] * a.ndim
    src[axis] = slice(None, n // 2)
    dst[axis] = slice(None, n // 2)
    out[tuple(dst)] = a[tuple(src)]
    src[axis] = slice(N - n // 2 + 1, None)
    dst[axis] = slice(n // 2, None)
    out[tuple(dst)] = a[tuple(src)]
    return out


def zeropad_rfft(a: np.ndarray, n: int) -> np.ndarray:
    """fft.py:140-163: append zeros on the last (kx) axis."""
    N = a.shape[-1]
    out = np.zeros(a.shape[:-1] + (n,), dtype=a.dtype)
    out[..., :N] = a
    return out


def truncate_rfft(a: np.ndarray, n: int) -> np.ndarray:
    """fft.py:166-190: keep the lowest n non-negative kx modes."""
    return np.ascontiguousarray(a[..., :n])


def rfft3d(x: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    """fft.py:291-348: physical [y,z,x] -> spectral [ky,kz,kx], x->z->y."""
    y = truncate_rfft(parallel.fft(np.fft.rfft, x, 2, norm=NORM), nx // 2)
    y = truncate_fft(parallel.fft(np.fft.fft, y, 1, norm=NORM), nz, 1)
    y = truncate_fft(parallel.fft(np.fft.fft, y, 0, norm=NORM), ny, 0)
    return y


def irfft3d(x: np.ndarray, nx_p: int, ny_p: int, nz_p: int) -> np.ndarray:
    """fft.py:351-408: spectral [ky,kz,kx] -> physical [y,z,x], y->z->x."""
    y = parallel.fft(np.fft.ifft, zeropad_fft(x, ny_p, 0), 0, norm=NORM)
    y = parallel.fft(np.fft.ifft, zeropad_fft(y, nz_p, 1), 1, norm=NORM)
    y = zeropad_rfft(y, nx_p // 2 + 1)
    return parallel.fft(np.fft.irfft, y, 2, norm=NORM)


def rfft2d(x: np.ndarray, nx: int, nz: int) -> np.ndarray:
    """fft.py:193-240: physical [y,z,x] -> [y,kz,kx], x then z."""
    y = truncate_rfft(parallel.fft(np.fft.rfft, x, 2, norm=NORM), nx // 2)
    return truncate_fft(parallel.fft(np.fft.fft, y, 1, norm=NORM), nz, 1)


def irfft2d(x: np.ndarray, nx_p: int, nz_p: int) -> np.ndarray:
    """fft.py:243-288: [y,kz,kx] -> physical [y,z,x], z then x."""
    y = parallel.fft(np.fft.ifft, zeropad_fft(x, nz_p, 1), 1, norm=NORM)
    y = zeropad_rfft(y, nx_p // 2 + 1)
    return parallel.fft(np.fft.irfft, y, 2, norm=NORM)


# operators.py:59-146: vmapped wrappers over the 3 velocity components.
def phys_to_spec(v: np.ndarray, cfg) -> np.ndarray:
    return np.stack([rfft3d(c, cfg.nx, cfg.ny, cfg.nz) for c in v])


def spec_to_phys(v: np.ndarray, cfg) -> np.ndarray:
    return np.stack(
        [irfft3d(c, cfg.nx_padded, cfg.ny_padded, cfg.nz_padded) for c in v]
    )


def phys_to_spec_2d(v: np.ndarray, cfg) -> np.ndarray:
    """operators.py:104-124: output transposed to [kz,kx,y]."""
    return np.stack(
        [np.transpose(rfft2d(c, cfg.nx, cfg.nz), (1, 2, 0)) for c in v]
    )


def spec_to_phys_2d(v: np.ndarray, cfg) -> np.ndarray:
    """operators.py:127-146: input [kz,kx,y] transposed to [y,kz,kx]."""
    return np.stack(
        [
            irfft2d(np.transpose(c, (2, 0, 1)), cfg.nx_padded, cfg.nz_padded)
            for c in v
        ]
    )


def cross(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """operators.py:149-173."""
    return np.array(
        [
            a[1] * b[2] - a[2] * b[1],
            a[2] * b[0] - a[0] * b[2],
            a[0] * b[1] - a[1] * b[0],
        ]
    )


def real_harmonics(n: int) -> np.ndarray:
    """operators.py:18-34: [0, 1, ..., n/2-1]."""
    return np.arange(0, n // 2, dtype=int)


def complex_harmonics(n: int) -> np.ndarray:
    """operators.py:37-56: FFT order with the Nyquist mode omitted."""
    qs = (np.arange(n, dtype=int) + n // 2) % n - n // 2
    out = np.zeros(n - 1, dtype=int)
    out[: n // 2] = qs[: n // 2]
    out[n // 2 :] = qs[n // 2 + 1 :]
    return out


def get_nonlin(velocity_spec, base_flow, curl_base_flow, nonlin_base_flow,
               to_phys, to_spec, curl_fn):
    """rhs.py:34-92: rotational-form nonlinear term on the padded grid."""
    velocity_phys = to_phys(velocity_spec)
    vorticity_phys = to_phys(curl_fn(velocity_spec))
    nonlin_phys = cross(velocity_phys, vorticity_phys)
    nonlin_phys = nonlin_phys + (
        cross(velocity_phys, curl_base_flow)
        + cross(base_flow, vorticity_phys)
        + nonlin_base_flow
    )
    return to_spec(nonlin_phys)
