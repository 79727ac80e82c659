"""Poisson's equation on an `IonOpticsMesh` with a Boltzmann plasma species, on the B200.

The interface of the reference's ``solver/poisson.py`` (``IonOpticsPoisson``,
``BoltzmannElectrons``, ``BoltzmannIons``; ``poisson.py:54-141, 536-933``).  The operator
is the finite-volume Laplacian of the reference's field (5-point rows, Shortley--Weller
rows next to electrodes, ``(1 -/+ 1/2j)`` radial weights, ``4 (phi_1 - phi_0)`` on the axis,
mirror images on Neumann faces), built and solved on the device by
``libbt200.so``: GMRES preconditioned by a geometric multigrid V-cycle, and for a plasma
Newton's method whose every step solves its own Jacobian (the multigrid rebuilt for it).
"""

from __future__ import annotations

import ctypes
from collections.abc import Callable
from dataclasses import dataclass
from typing import Any

import numpy as np

from beamtracer_b200 import _lib
from beamtracer_b200.mesh import FACES, IonOpticsMesh

#: The linear solves' relative residual (the reference factorises exactly with LU).
LINEAR_TOLERANCE = 1e-13


@dataclass(frozen=True)
class BoltzmannElectrons:
    """Plasma electrons for positive-ion extraction: ``-rho_e exp((phi - U_p) / T_e)``
    (``poisson.py:54-94``); ``rho_e`` [C/m^3], ``electron_temperature`` [eV],
    ``plasma_potential`` [V]."""

    rho_e: float
    electron_temperature: float
    plasma_potential: float
    sign = -1

    @property
    def density(self) -> float:
        return self.rho_e

    @property
    def temperature(self) -> float:
        return self.electron_temperature


@dataclass(frozen=True)
class BoltzmannIons:
    """Plasma positive ions for negative-ion extraction: ``rho_p exp(-(phi - U_p) / T_p)``
    (``poisson.py:97-141``)."""

    rho_p: float
    ion_temperature: float
    plasma_potential: float
    sign = 1

    @property
    def density(self) -> float:
        return self.rho_p

    @property
    def temperature(self) -> float:
        return self.ion_temperature


def _neumann_values(mesh: IonOpticsMesh) -> np.ndarray:
    values = np.zeros(4)
    for k, face in enumerate(FACES):
        condition = mesh.faces[face]
        if condition.kind != "neumann":
            continue
        if callable(condition.value):
            raise NotImplementedError(
                f"a Neumann condition that varies along the face ({face}) is not supported"
            )
        values[k] = float(condition.value)
    return values


class IonOpticsPoisson:
    """Solve ``laplace(phi) = -rho / epsilon_0`` (plus a Boltzmann species) on a mesh.

    ``backend`` is accepted for the reference's signature; every backend is the device's
    multigrid-preconditioned GMRES.  With refined boxes (``refinement``, linear solves) the
    potential and charge density live on the composite nodes of `layout`
    (`beamtracer_b200.composite.CompositePoisson`).  A distributed solve (``comm``) is not
    part of this build.  ``homogeneous`` zeroes the held values and face terms (the
    corrections of the composite solve).
    """

    def __init__(
        self,
        mesh: IonOpticsMesh,
        reuse_jacobian: bool = True,
        backend: str = "multigrid",
        comm: Any = None,
        refinement=(),
        *,
        transposed: bool = False,
        homogeneous: bool = False,
    ) -> None:
        self.mesh = mesh
        self.reuse_jacobian = bool(reuse_jacobian)
        self.backend = backend
        self.comm = comm
        self.refinement = tuple(refinement)
        self._layout = None
        self._composite = None
        if self.refinement:
            if transposed:
                raise NotImplementedError("the transposed solver takes no refined boxes")
            from beamtracer_b200.composite import CompositePoisson
            from beamtracer_b200.refinement import layout_of_mesh

            self._layout = layout_of_mesh(mesh, self.refinement)
            self._composite = CompositePoisson(self._layout)
        #: Newton steps, V-cycles of the last solve (the reference's factorisations and
        #: Krylov steps have no counterpart: every step is a Krylov solve).
        self.newton_iterations = 0
        self.factorisations = 0
        self.krylov_steps = 0
        self._ctx = _lib.context()
        nx, ny = mesh.shape
        self._fixed = np.ascontiguousarray(mesh.fixed, dtype=np.uint8)
        self._value = np.ascontiguousarray(mesh.fixed_value, dtype=np.float64)
        self._distance = np.ascontiguousarray(mesh.distance, dtype=np.float64)
        self._x = np.ascontiguousarray(mesh.x, dtype=np.float64)
        self._neumann = _neumann_values(mesh)
        #: a solver of the transposed free block A_ff^T z = b (held values and face terms
        #: zero), for the adjoint; linear solves only
        self.transposed = bool(transposed)
        if self.transposed or homogeneous:
            self._value = np.zeros_like(self._value)
            self._neumann = np.zeros_like(self._neumann)
        desc = _lib.MeshDesc(
            nx, ny, float(mesh.h), self._x.ctypes.data, float(mesh.origin[1]),
            int(mesh.cylindrical), self._fixed.ctypes.data, self._value.ctypes.data,
            self._distance.ctypes.data, self._neumann.ctypes.data,
        )  # fmt: skip
        handle = _lib.P()
        _lib.check(_lib.lib().bt_poisson_create(self._ctx.handle, ctypes.byref(desc),
                                                ctypes.byref(handle)))  # fmt: skip
        self._handle = handle
        self._region_key: object = None
        if self.transposed:
            _lib.check(_lib.lib().bt_poisson_set_transposed(handle, 1))

    @property
    def layout(self):
        """The composite nodes the potential lives on (the mesh's own nodes without refined
        boxes; ``poisson.py:611-616``)."""
        if self._layout is None:
            from beamtracer_b200.refinement import layout_of_mesh

            self._layout = layout_of_mesh(self.mesh)
        return self._layout

    @property
    def coordinates(self) -> np.ndarray:
        """The positions of the composite nodes, ``(2, nodes)`` [m]: ``(x, y)``, or
        ``(x, r)`` in cylindrical geometry (``poisson.py:617-625``)."""
        layout = self.layout
        return np.ascontiguousarray(np.stack([layout.x, layout.y]))

    def fixed_adjoint(self, z, phi_bar, out) -> None:
        """``out`` (device, (nx, ny)) <- the sensitivity to the held nodes' potentials of a
        quantity whose sensitivity to the potential is ``phi_bar``, given
        ``z = A_ff^-T phi_bar`` on the free nodes (``bt_poisson_fixed_adjoint``)."""
        _lib.check(_lib.lib().bt_poisson_fixed_adjoint(self._handle, _lib.dptr(z),
                                                       _lib.dptr(phi_bar), _lib.dptr(out)))  # fmt: skip

    def rebind(self, ctx) -> None:
        """Queue this solver's later work on the library context ``ctx`` (same device)."""
        if ctx is self._ctx:
            return
        _lib.check(_lib.lib().bt_poisson_set_context(self._handle, ctx.handle))
        self._ctx = ctx

    def close(self) -> None:
        if getattr(self, "_composite", None) is not None:
            self._composite.close()
            self._composite = None
        if getattr(self, "_handle", None):
            _lib.lib().bt_poisson_destroy(self._handle)
            self._handle = None

    def __del__(self) -> None:  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def set_options(self, fine_sweeps: int = 2, coarse_sweeps: int = 2, staged: bool = True,
                    tail_nodes: int = 4096) -> None:
        """The V-cycle's settings: red-black sweeps on the finest level, four-colour sweeps
        on the coarse levels, smoothing staged through shared memory or one launch per
        colour (the same values), and the largest level the one-block tail may take."""
        _lib.check(_lib.lib().bt_poisson_set_options(self._handle, int(fine_sweeps),
                                                     int(coarse_sweeps), int(bool(staged)),
                                                     int(tail_nodes)))  # fmt: skip

    # -- the device path --------------------------------------------------------------

    def hold(self, region: Any, potential: float = 0.0) -> None:
        """Hold the nodes of ``region`` (an (nx, ny) mask, a function of the nodes'
        ``(x, y)``, or None for none) that the mesh does not fix at ``potential`` in later
        solves (the initial plasma region; a refined box's sides in its corrections); a
        region equal to the one held already changes nothing."""
        self._set_region(region, potential)

    def _set_region(self, region: Any, potential: float) -> None:
        if region is None:
            key: object = None
        elif callable(region):
            key = (id(region), float(potential))
        else:
            key = (np.packbits(np.asarray(region, dtype=bool)).tobytes(), float(potential))
        if key == self._region_key:
            return
        mask = None
        if region is not None:
            if callable(region):
                x, y = self.mesh.nodes()
                mask = np.asarray(region(x, y), dtype=bool)
            else:
                mask = np.asarray(region, dtype=bool)
            if mask.shape != self.mesh.shape:
                raise ValueError("the fixed region needs the mesh's shape")
            mask = np.ascontiguousarray(mask, dtype=np.uint8)
        _lib.check(
            _lib.lib().bt_poisson_set_region(
                self._handle, None if mask is None else mask.ctypes.data, float(potential)
            )
        )
        self._region_key = key

    def solve_device(
        self,
        phi,
        rho=None,
        *,
        plasma: BoltzmannElectrons | BoltzmannIons | None = None,
        fixed_region: np.ndarray | Callable | None = None,
        fixed_potential: float = 0.0,
        tolerance: float = 1.0e-6,
        max_newton: int = 100,
        linear_tolerance: float = LINEAR_TOLERANCE,
    ) -> None:
        """Solve in place on device arrays: ``phi`` (nx, ny) float64 holds the first guess
        and receives the potential; ``rho`` (nx, ny) float64 [C/m^3] or None.

        With ``plasma`` Newton's method stops when its largest update is below
        ``tolerance * max(ptp(prescribed potentials), T, 1 V)`` (``poisson.py:874-877``).
        """
        if self._composite is not None:
            species, newton_tol = None, 0.0
            if plasma is not None:
                layout = self._layout
                prescribed = layout.fixed_value[layout.fixed]
                scale = max(float(np.ptp(prescribed)) if prescribed.size else 0.0,
                            float(plasma.temperature), 1.0)  # fmt: skip
                from scipy.constants import epsilon_0

                species = (float(plasma.density) / epsilon_0, float(plasma.temperature),
                           float(plasma.plasma_potential), int(plasma.sign))  # fmt: skip
                newton_tol = float(tolerance) * scale
            self._composite.solve_device(phi, rho, fixed_region=fixed_region,
                                         fixed_potential=fixed_potential, plasma=species,
                                         newton_tolerance=newton_tol, max_newton=max_newton)  # fmt: skip
            self.newton_iterations = self._composite.newton_iterations
            self.krylov_steps = self._composite.krylov_steps
            return
        self._set_region(fixed_region, fixed_potential)
        if self.transposed and (plasma is not None or fixed_region is not None):
            raise NotImplementedError("the transposed solver takes linear solves only")
        steps, cycles = _lib.I32(), _lib.I32()
        if plasma is None:
            args = (0.0, 1.0, 0.0, 1, linear_tolerance, 0.0, 0)
        else:
            prescribed = self._value[self._fixed.astype(bool)]
            scale = max(float(np.ptp(prescribed)) if prescribed.size else 0.0,
                        float(plasma.temperature), 1.0)  # fmt: skip
            from scipy.constants import epsilon_0

            args = (
                float(plasma.density) / epsilon_0, float(plasma.temperature),
                float(plasma.plasma_potential), int(plasma.sign), 1e-6,
                float(tolerance) * scale, int(max_newton),
            )  # fmt: skip
        _lib.check(
            _lib.lib().bt_poisson_solve(
                self._handle, _lib.dptr(phi), _lib.dptr(rho), *args,
                ctypes.byref(steps), ctypes.byref(cycles),
            )
        )  # fmt: skip
        self.newton_iterations = steps.value if plasma is not None else 0
        self.krylov_steps = cycles.value
        self.factorisations = 0

    # -- the reference's host interface ------------------------------------------------

    def solve(
        self,
        rho: np.ndarray | None = None,
        *,
        plasma: BoltzmannElectrons | BoltzmannIons | None = None,
        fixed_region: np.ndarray | Callable | None = None,
        fixed_potential: float = 0.0,
        initial: np.ndarray | None = None,
        tolerance: float = 1.0e-6,
        max_newton: int = 100,
    ) -> np.ndarray:
        """The potential (nx, ny) for the charge density ``rho`` [C/m^3] (host arrays).

        Without ``initial`` a plasma's Newton iteration starts from the linear solution, as
        the reference's starts from its vacuum solution (``poisson.py:843-860``).
        """
        import torch

        shape = self.mesh.shape if self._composite is None else (self._layout.size,)
        phi = torch.zeros(shape, dtype=torch.float64, device="cuda")
        rho_dev = None
        if rho is not None:
            rho = np.asarray(rho, dtype=np.float64)
            if rho.shape != shape:
                raise ValueError(f"rho needs the shape {shape} (the mesh's, or the refined "
                                 "layout's composite nodes)")
            rho_dev = torch.from_numpy(np.ascontiguousarray(rho)).cuda()
        if initial is not None:
            phi.copy_(torch.from_numpy(np.ascontiguousarray(initial, dtype=np.float64)))
        if plasma is None or initial is None:
            self.solve_device(phi, rho_dev, fixed_region=fixed_region,
                              fixed_potential=fixed_potential)  # fmt: skip
        if plasma is not None:
            self.solve_device(phi, rho_dev, plasma=plasma, fixed_region=fixed_region,
                              fixed_potential=fixed_potential, tolerance=tolerance,
                              max_newton=max_newton)  # fmt: skip
        return phi.cpu().numpy()
