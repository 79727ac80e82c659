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


def surface_field_device(mesh: IonOpticsMesh, field: StaggeredElectricField,
                         arrays: MeshArrays | None = None):
    """``(magnitude, electrode, largest)`` on the device: |E| at the free nodes next to an
    electrode (NaN elsewhere), that electrode (-1 elsewhere) and every electrode's largest
    |E| (``bt_surface_field``)."""
    import torch

    arrays = arrays or MeshArrays(mesh)
    nx, ny = mesh.shape
    magnitude = torch.empty((nx, ny), dtype=torch.float64, device="cuda")
    electrode = torch.empty((nx, ny), dtype=torch.int32, device="cuda")
    count = len(mesh.electrodes)
    largest = torch.zeros(max(count, 1), dtype=torch.float64, device="cuda")
    ctx = _lib.context()
    _lib.check(_lib.lib().bt_surface_field(
        ctx.handle, _lib.dptr(field.fx_device), _lib.dptr(field.fy_device),
        _lib.dptr(arrays.solid), _lib.dptr(arrays.near), nx, ny, count, _lib.dptr(magnitude),
        _lib.dptr(electrode), _lib.dptr(largest)))  # fmt: skip
    return magnitude, electrode, largest[:count]


def surface_field(mesh: IonOpticsMesh, field: StaggeredElectricField
                  ) -> tuple[np.ndarray, np.ndarray]:  # fmt: skip
    """|E| [V/m] at the free nodes next to an electrode and that electrode, both of the
    mesh's shape (NaN and -1 elsewhere): the interface of ``fields.py:324-377``, computed
    on the device.  The component along an axis with an electrode neighbour is the edge
    towards it, taken over the bracketed distance to the surface (the field at the
    surface).  At a sharp corner the field is singular and grows as the mesh is refined."""
    magnitude, electrode, _ = surface_field_device(mesh, field)
    return magnitude.cpu().numpy(), electrode.cpu().numpy()


def _derivative_weights() -> np.ndarray:
    """(7, 7) weights of the central differences over the samples ``i - 3 .. i + 3``: row
    ``k`` gives ``h^k d^k B / dz^k`` -- orders 6, 6, 4, 4, 2, 2 for ``k = 1 .. 6`` (the widest
    central stencil of each derivative that seven points hold), the sample itself for 0."""
    rows = {
        0: ((0, 0, 0, 1, 0, 0, 0), 1),
        1: ((-1, 9, -45, 0, 45, -9, 1), 60),
        2: ((2, -27, 270, -490, 270, -27, 2), 180),
        3: ((1, -8, 13, 0, -13, 8, -1), 8),
        4: ((-1, 12, -39, 56, -39, 12, -1), 6),
        5: ((-1, 4, -5, 0, 5, -4, 1), 2),
        6: ((1, -6, 15, -20, 15, -6, 1), 1),
    }  # fmt: skip
    return np.array([np.array(num, dtype=float) / den for num, den in (rows[k] for k in range(7))])


class AxisymmetricMagneticField:
    """A static axisymmetric magnetic field from its on-axis profile (the interface of
    ``fields.py:192-279``).

    ``bz`` [T] sampled at ``z0 + hz k``.  The derivatives ``B^(k)`` of the profile, to
    ``order`` (at most 6), are central differences over seven samples at every sample with
    three neighbours on each side (zero at the three end samples), interpolated linearly
    between samples and extrapolated along the first and last valid cells.  Off the axis
    the fields are the current-free series

        B_z = sum_k (-1)^k (r/2)^(2k) B^(2k) / (k!)^2,
        B_r = sum_k (-1)^(k+1) (r/2)^(2k+1) B^(2k+1) / (k! (k+1)!),

    kept to the terms whose derivative order is at most ``order``.
    """

    def __init__(self, z0: float, hz: float, bz, order: int = 6) -> None:
        samples = np.asarray(bz, dtype=float)
        if samples.ndim != 1 or samples.size < 8:
            raise ValueError("the on-axis profile needs at least 8 samples")
        if not 0 <= order <= 6:
            raise ValueError(f"order must be 0 to 6, got {order}")
        self.z0, self.hz, self.order, self.bz = float(z0), float(hz), int(order), samples
        from numpy.lib.stride_tricks import sliding_window_view

        windows = sliding_window_view(samples, 7)  # (n - 6, 7), centred on samples 3 .. n - 4
        weights = _derivative_weights()[: self.order + 1]
        scale = self.hz ** -np.arange(self.order + 1, dtype=float)
        table = np.zeros((samples.size, self.order + 1))
        table[3:-3] = (windows @ weights.T) * scale
        #: (n, order + 1): d^k B_z / dz^k at every sample, a row per sample
        self._samples = np.ascontiguousarray(table)

    def derivatives(self, z) -> np.ndarray:
        """``(order + 1, len(z))``: the derivatives of the profile at ``z``."""
        s = (np.asarray(z, dtype=float) - self.z0) / self.hz
        cell = np.clip(np.floor(s).astype(np.int64), 3, self.bz.size - 5)
        t = (s - cell)[:, None]
        below, above = self._samples[cell], self._samples[cell + 1]
        return (below + t * (above - below)).T

    def __call__(self, z, r) -> tuple[np.ndarray, np.ndarray]:
        """``(B_z, B_r)`` [T] at axial positions ``z`` and radii ``r``."""
        from math import factorial

        d = self.derivatives(z)
        half = 0.5 * np.asarray(r, dtype=float)
        bz = np.zeros(d.shape[1])
        br = np.zeros(d.shape[1])
        for n in range(self.order + 1):  # the term of the n-th derivative
            k = n // 2
            if n % 2 == 0:
                bz = bz + ((-1) ** k / factorial(k) ** 2) * half ** (2 * k) * d[n]
            else:
                br = br + ((-1) ** (k + 1) / (factorial(k) * factorial(k + 1))) * half ** n * d[n]
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
    """The on-axis B_z [T] of a thin-walled solenoid (a finite current sheet of ``length``
    and winding ``radius``, centred at ``centre``), scaled to ``peak`` at its centre (the
    interface of ``fields.py:290-321``): proportional to the difference of the cosines of
    the angles under which the two ends are seen, ``cos(a1) - cos(a2)``."""
    z = np.asarray(z, dtype=float)

    def ends(at):
        near_end = at - (centre - 0.5 * length)
        far_end = at - (centre + 0.5 * length)
        return near_end / np.hypot(near_end, radius) - far_end / np.hypot(far_end, radius)

    return peak * ends(z) / ends(np.asarray(centre, dtype=float))
