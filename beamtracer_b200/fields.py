"""Fields for the trace: the staggered electric field, on the device, and the axisymmetric
magnetic field of an on-axis profile.

The interface of the reference's ``solver/fields.py``: ``StaggeredElectricField``
(``fields.py:90-166``), ``AxisymmetricMagneticField`` (``fields.py:192-279``) and
``solenoid_on_axis`` (``fields.py:290-321``).
"""

from __future__ import annotations

import ctypes
from collections.abc import Sequence

import numpy as np

from beamtracer_b200 import _lib
from beamtracer_b200.mesh import IonOpticsMesh


def default_extrapolation(mesh: IonOpticsMesh) -> list[str]:
    """Linear extrapolation on every face, mirror (E = 0) on the axis or a symmetry plane."""
    faces = ["extrapolate"] * 4
    if mesh.cylindrical or mesh.symmetry_plane:
        faces[2] = "symmetric"
    return faces


class MeshArrays:
    """The device copies of a mesh's classification that the edge field reads."""

    def __init__(self, mesh: IonOpticsMesh) -> None:
        import torch

        self.mesh = mesh
        self.solid = torch.from_numpy(np.ascontiguousarray(mesh.solid, dtype=np.int32)).cuda()
        self.near = torch.from_numpy(np.ascontiguousarray(mesh.near_solid, dtype=np.uint8)).cuda()
        self.distance = torch.from_numpy(np.ascontiguousarray(mesh.distance)).cuda()
        self.dx = torch.from_numpy(np.ascontiguousarray(mesh.dx)).cuda() if mesh.graded else None


class StaggeredElectricField:
    """The electric field of a potential on the edges between nodes (``fields.py:90-166``).

    ``E_x`` on the (nx + 1, ny) edges along x, ``E_y`` on the (nx, ny + 1) edges along y,
    built on the device from ``potential`` (a host array or a device array) and
    interpolated bilinearly at points.  ``fx_device``, ``fy_device`` are the device arrays;
    ``fx``, ``fy`` host copies (made when asked for).
    """

    def __init__(
        self,
        mesh: IonOpticsMesh,
        potential,
        extrapolation: Sequence[str] | None = None,
        *,
        arrays: MeshArrays | None = None,
        out=None,
    ) -> None:
        import torch

        self.mesh = mesh
        self.extrapolation = tuple(extrapolation or default_extrapolation(mesh))
        for face in self.extrapolation:
            if face not in ("extrapolate", "symmetric"):
                raise ValueError(f"unknown face extrapolation {face!r}")
        arrays = arrays or MeshArrays(mesh)
        nx, ny = mesh.shape
        if _lib.is_device_array(potential):
            phi = potential
        else:
            phi = torch.from_numpy(np.ascontiguousarray(potential, dtype=np.float64)).cuda()
        if tuple(phi.shape) != (nx, ny):
            raise ValueError("the potential needs the mesh's shape")
        if out is None:
            fx = torch.empty((nx + 1, ny), dtype=torch.float64, device="cuda")
            fy = torch.empty((nx, ny + 1), dtype=torch.float64, device="cuda")
        else:
            fx, fy = out
        faces = (ctypes.c_int32 * 4)(*[int(f == "symmetric") for f in self.extrapolation])
        ctx = _lib.context()
        _lib.check(
            _lib.lib().bt_edge_field(
                ctx.handle, _lib.dptr(phi), _lib.dptr(arrays.solid), _lib.dptr(arrays.near),
                _lib.dptr(arrays.distance), _lib.dptr(arrays.dx), nx, ny, float(mesh.h),
                faces, _lib.dptr(fx), _lib.dptr(fy),
            )
        )  # fmt: skip
        self.fx_device, self.fy_device = fx, fy

    @property
    def fx(self) -> np.ndarray:
        return self.fx_device.cpu().numpy()

    @property
    def fy(self) -> np.ndarray:
        return self.fy_device.cpu().numpy()

    def __call__(self, x, y) -> tuple[np.ndarray, np.ndarray]:
        """``(E_x, E_y)`` [V/m] at the points ``(x, y)`` (host arrays), gathered on the device."""
        import torch

        from beamtracer_b200.kernels import staggered_field_2d

        mesh = self.mesh
        x = np.ascontiguousarray(x, dtype=float).ravel()
        y = np.ascontiguousarray(y, dtype=float).ravel()
        if not x.size:
            return np.empty(0), np.empty(0)
        px = torch.from_numpy(np.ascontiguousarray(mesh.logical_x(x))).cuda()
        py = torch.from_numpy(y).cuda()
        ex = torch.empty_like(px)
        ey = torch.empty_like(px)
        staggered_field_2d(px, py, self.fx_device, self.fy_device, *map(float, mesh.logical_origin),
                           mesh.h, ex, ey)  # fmt: skip
        return ex.cpu().numpy(), ey.cpu().numpy()


class AxisymmetricMagneticField:
    """A static axisymmetric magnetic field from its on-axis profile (``fields.py:192-279``).

    ``bz`` [T] sampled at ``z0 + hz k``; off the axis the power series in ``r`` to ``order``
    (at most 6) with 7-point finite-difference derivatives of the profile, linearly
    interpolated between the samples.
    """

    #: The derivative stencils (orders 6, 6, 4, 4, 2, 2 for derivatives 1..6).
    STENCILS = (
        (0, 0, 0, 1, 0, 0, 0),
        (-1 / 60, 9 / 60, -45 / 60, 0, 45 / 60, -9 / 60, 1 / 60),
        (2 / 180, -27 / 180, 270 / 180, -490 / 180, 270 / 180, -27 / 180, 2 / 180),
        (1 / 8, -8 / 8, 13 / 8, 0, -13 / 8, 8 / 8, -1 / 8),
        (-1 / 6, 12 / 6, -39 / 6, 56 / 6, -39 / 6, 12 / 6, -1 / 6),
        (-1 / 2, 4 / 2, -5 / 2, 0, 5 / 2, -4 / 2, 1 / 2),
        (1, -6, 15, -20, 15, -6, 1),
    )

    def __init__(self, z0: float, hz: float, bz, order: int = 6) -> None:
        samples = np.asarray(bz, dtype=float)
        if samples.ndim != 1 or samples.size < 8:
            raise ValueError("the on-axis profile needs at least 8 samples")
        if not 0 <= order <= 6:
            raise ValueError(f"order must be 0 to 6, got {order}")
        self.z0, self.hz, self.order, self.bz = float(z0), float(hz), int(order), samples
        n = samples.size
        centre = np.arange(3, n - 3)
        self._derivatives = np.zeros((self.order + 1, n))
        for k, stencil in enumerate(self.STENCILS[: self.order + 1]):
            d = sum(c * samples[centre + a - 3] for a, c in enumerate(stencil))
            self._derivatives[k, centre] = d / self.hz**k
        self._samples = np.ascontiguousarray(self._derivatives.T)

    def derivatives(self, z) -> np.ndarray:
        n = self.bz.size
        s = (np.asarray(z, dtype=float) - self.z0) / self.hz
        i = np.clip(np.floor(s).astype(np.int64), 3, n - 5)
        t = (s - i)[:, None]
        low = self._samples[i]
        return (low + t * (self._samples[i + 1] - low)).T

    def __call__(self, z, r) -> tuple[np.ndarray, np.ndarray]:
        d = self.derivatives(z)
        r = np.asarray(r, dtype=float)
        r2 = r * r
        bz_c = (1.0, -1.0 / 4.0, 1.0 / 64.0, -1.0 / 2304.0)
        br_c = (-1.0 / 2.0, 1.0 / 16.0, -1.0 / 384.0)
        bz = d[0].copy()
        br = np.zeros_like(bz)
        power = np.ones_like(r2)
        for k in range(1, self.order // 2 + 1):
            power = power * r2
            bz += bz_c[k] * power * d[2 * k]
        power = r.copy()
        for k in range((self.order + 1) // 2):
            br += br_c[k] * power * d[2 * k + 1]
            power = power * r2
        return bz, br

    def profile(self) -> MagneticProfile:
        """The field on the device for a cylindrical mesh (``B_z`` along x, ``B_r``)."""
        return MagneticProfile(1, self, 0.0)

    @property
    def samples(self) -> np.ndarray:
        """The derivative table ``(n, order + 1)``: ``d^k B_z / dz^k`` at every sample."""
        return self._samples


class PlanarSolenoidField:
    """A solenoid's axisymmetric field laid on a planar mesh, its axis the line
    ``y = axis_y``: ``(B_x, B_y, B_z) = (B_z, sign(y - axis_y) B_r, 0)`` at
    ``r = |y - axis_y|`` -- the magnetic callable ``BeamTracer`` takes on a planar mesh
    (``tracer.py:401-404, 567-572``), built from `AxisymmetricMagneticField`."""

    def __init__(self, field: AxisymmetricMagneticField, axis_y: float = 0.0) -> None:
        self.field = field
        self.axis_y = float(axis_y)

    def __call__(self, x, y) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        y = np.asarray(y, dtype=float)
        yr = y - self.axis_y
        bz, br = self.field(x, np.abs(yr))
        return bz, np.where(yr < 0.0, -br, br), np.zeros_like(bz)

    def profile(self) -> MagneticProfile:
        return MagneticProfile(2, self.field, self.axis_y)


class MagneticProfile:
    """An on-axis profile's derivative table on the device, for the magnetic trace
    (``bt_magnetic``): mode 1 on a cylindrical mesh, 2 on a planar one."""

    def __init__(self, mode: int, field: AxisymmetricMagneticField, axis_y: float) -> None:
        import torch

        self.mode = int(mode)
        self.order = field.order
        self.z0, self.hz, self.axis_y = field.z0, field.hz, float(axis_y)
        self.samples = torch.from_numpy(np.ascontiguousarray(field.samples)).to("cuda")

    def descriptor(self) -> _lib.MagneticDesc:
        return _lib.MagneticDesc(self.mode, self.order, int(self.samples.shape[0]), self.z0,
                                 self.hz, self.axis_y, _lib.dptr(self.samples))  # fmt: skip

    def oracle_tuple(self) -> tuple:
        """``(mode, order, z0, hz, axis_y, samples)`` for the oracle."""
        return (self.mode, self.order, self.z0, self.hz, self.axis_y,
                self.samples.cpu().numpy())  # fmt: skip


def solenoid_on_axis(z, centre: float, length: float, radius: float, peak: float) -> np.ndarray:
    """The on-axis B_z [T] of a thin-walled solenoid scaled to ``peak`` at its centre
    (``fields.py:307-321``)."""
    z = np.asarray(z, dtype=float)

    def shape(zz):
        a = zz - centre + 0.5 * length
        b = zz - centre - 0.5 * length
        return a / np.hypot(a, radius) - b / np.hypot(b, radius)

    return peak * shape(z) / shape(np.asarray(centre))
