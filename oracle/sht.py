"""FP64 restatement of dinosaur's Real spherical-harmonic basis and operators.

Test infrastructure (see ``oracle/__init__.py``).  Follows
``dinosaur/associated_legendre.py``, ``dinosaur/fourier.py`` and the
``RealSphericalHarmonics`` / ``Grid`` classes of
``dinosaur/spherical_harmonic.py`` (reference v1.3.6).

Layouts match the reference: nodal arrays are ``[..., lon, lat]`` with latitude
fastest and Gauss nodes ascending in sin(latitude); modal arrays are
``[..., m, l]`` with rows ordered m = 0, +1, -1, +2, -2, ... (cos, sin).
"""

from __future__ import annotations

import dataclasses
import functools
import math

import numpy as np
import scipy.special


# ---------------------------------------------------------------------------
# Quadrature nodes
# ---------------------------------------------------------------------------

def gauss_legendre_nodes(n: int) -> tuple[np.ndarray, np.ndarray]:
  """Gauss-Legendre nodes/weights, ascending (associated_legendre.py:104-114)."""
  return scipy.special.roots_legendre(n)


def _weights_for_nodes(x: np.ndarray) -> np.ndarray:
  """Quadrature weights exact for Legendre polynomials up to len(x)-1.

  Follows associated_legendre.py:160-175: solve sum_j w_j P_k(x_j) = delta_k0
  and normalise the weights to sum to 2.
  """
  legendre = legendre_table(1, x.shape[0], x)[0].T
  z = np.zeros_like(x)
  z[0] = 1
  w = np.linalg.solve(legendre, z)
  return w / w.sum() * 2


def equiangular_nodes(n: int) -> tuple[np.ndarray, np.ndarray]:
  """Cell-centred equiangular latitudes (associated_legendre.py:117-137)."""
  spacing = np.pi / n
  theta = np.linspace(-np.pi / 2 + spacing / 2, np.pi / 2 - spacing / 2, n)
  x = np.sin(theta)
  return x, _weights_for_nodes(x)


def equiangular_nodes_with_poles(n: int) -> tuple[np.ndarray, np.ndarray]:
  """Equiangular latitudes including the poles (associated_legendre.py:140-157)."""
  theta = np.linspace(-np.pi / 2, np.pi / 2, n)
  x = np.sin(theta)
  return x, _weights_for_nodes(x)


LATITUDE_SPACINGS = dict(
    gauss=gauss_legendre_nodes,
    equiangular=equiangular_nodes,
    equiangular_with_poles=equiangular_nodes_with_poles,
)


# ---------------------------------------------------------------------------
# Basis functions
# ---------------------------------------------------------------------------

def legendre_table(n_m: int, n_l: int, x: np.ndarray) -> np.ndarray:
  """Unit-L2[-1,1]-normalised associated Legendre functions p[m, j, l].

  Restates associated_legendre.py:23-101.  The diagonal is seeded with
  P_m^m = -sqrt(1 + 1/(2m)) * sqrt(1-x^2) * P_{m-1}^{m-1} (P_0^0 = 1/sqrt 2)
  and climbed in k = l - m with the normalised three-term recurrence
  p_k = a * (x p_{k-1} - b p_{k-2}).  Entries with l < m are zero.
  """
  if n_m > n_l:
    raise ValueError(f'Expected n_m <= n_l; got n_m = {n_m} and n_l = {n_l}.')
  x = np.asarray(x, dtype=np.float64)
  y = np.sqrt(1 - x * x)
  out = np.zeros((n_m, len(x), n_l))
  diag = np.full(len(x), 1 / np.sqrt(2))
  for m in range(n_m):
    if m > 0:
      diag = -np.sqrt(1 + 1 / (2 * m)) * y * diag
    prev2 = np.zeros(len(x))
    prev1 = diag
    out[m, :, m] = diag
    for k in range(1, n_l - m):
      mk2 = (m + k) ** 2
      mkp2 = (m + k - 1) ** 2
      a = np.sqrt((4 * mk2 - 1) / (mk2 - m * m))
      b = np.sqrt((mkp2 - m * m) / (4 * mkp2 - 1))
      cur = a * (x * prev1 - b * prev2)
      out[m, :, m + k] = cur
      prev2, prev1 = prev1, cur
  return out


def real_fourier_basis(wavenumbers: int, nodes: int) -> np.ndarray:
  """Real Fourier basis f[i, k] with unit L2[0,2pi) norm (fourier.py:24-60)."""
  if nodes < wavenumbers:
    raise ValueError(
        '`real_basis` requires nodes >= wavenumbers; '
        f'got m = {nodes} and n = {wavenumbers}.')
  lam = 2 * np.pi * np.arange(nodes) / nodes
  f = np.empty((nodes, 2 * wavenumbers - 1))
  f[:, 0] = 1 / np.sqrt(2 * np.pi)
  j = np.arange(1, wavenumbers)
  f[:, 1::2] = np.cos(np.outer(lam, j)) / np.sqrt(np.pi)
  f[:, 2::2] = np.sin(np.outer(lam, j)) / np.sqrt(np.pi)
  return f


def real_basis_derivative(u: np.ndarray, axis: int = -1) -> np.ndarray:
  """d/dlambda in the real Fourier basis (fourier.py:63-88)."""
  u = np.moveaxis(np.asarray(u), axis, -1)
  n = u.shape[-1]
  if n % 2 != 1:
    raise ValueError(f'{u.shape=} along {axis=} is not odd')
  out = np.zeros_like(u)
  j = np.arange(1, (n + 1) // 2)
  out[..., 2 * j - 1] = j * u[..., 2 * j]
  out[..., 2 * j] = -j * u[..., 2 * j - 1]
  return np.moveaxis(out, -1, axis)


def _shift(x: np.ndarray, offset: int, axis: int) -> np.ndarray:
  """Zero-padded roll (jax_numpy_utils.py:158-168)."""
  out = np.zeros_like(x)
  n = x.shape[axis]
  if abs(offset) >= n:
    return out
  src = [slice(None)] * x.ndim
  dst = [slice(None)] * x.ndim
  if offset > 0:
    src[axis] = slice(0, n - offset)
    dst[axis] = slice(offset, n)
  else:
    src[axis] = slice(-offset, n)
    dst[axis] = slice(0, n + offset)
  out[tuple(dst)] = x[tuple(src)]
  return out


# ---------------------------------------------------------------------------
# Grid
# ---------------------------------------------------------------------------

_CONSTANT_NORMALIZATION_FACTOR = 3.5449077  # spherical_harmonic.py:1154-1156


@dataclasses.dataclass(frozen=True)
class Grid:
  """FP64 Real-SH grid (spherical_harmonic.py:161-283, :678-1151)."""

  longitude_wavenumbers: int = 0
  total_wavenumbers: int = 0
  longitude_nodes: int = 0
  latitude_nodes: int = 0
  latitude_spacing: str = 'gauss'
  radius: float = 1.0
  # Arithmetic type of the transforms (float64 for the oracle; the CPU
  # baseline times the same contractions in float32).
  compute_dtype: type = np.float64

  @classmethod
  def construct(cls, max_wavenumber: int, gaussian_nodes: int, **kw) -> Grid:
    """spherical_harmonic.py:772-813."""
    return cls(max_wavenumber + 1, max_wavenumber + 2, 4 * gaussian_nodes,
               2 * gaussian_nodes, **kw)

  @classmethod
  def with_wavenumbers(cls, longitude_wavenumbers: int,
                       dealiasing: str = 'quadratic', **kw) -> Grid:
    """spherical_harmonic.py:737-770."""
    order = {'linear': 2, 'quadratic': 3, 'cubic': 4}[dealiasing]
    longitude_nodes = order * longitude_wavenumbers + 1
    latitude_nodes = math.ceil(longitude_nodes / 2)
    return cls(longitude_wavenumbers, longitude_wavenumbers + 1,
               longitude_nodes, latitude_nodes, **kw)

  # Standard grids (spherical_harmonic.py:833-917).
  @classmethod
  def T21(cls, **kw): return cls.construct(21, 16, **kw)
  @classmethod
  def T31(cls, **kw): return cls.construct(31, 24, **kw)
  @classmethod
  def T42(cls, **kw): return cls.construct(42, 32, **kw)
  @classmethod
  def T85(cls, **kw): return cls.construct(85, 64, **kw)
  @classmethod
  def TL31(cls, **kw): return cls.construct(31, 16, **kw)
  @classmethod
  def TL63(cls, **kw): return cls.construct(63, 32, **kw)
  @classmethod
  def TL127(cls, **kw): return cls.construct(127, 64, **kw)
  @classmethod
  def TL255(cls, **kw): return cls.construct(255, 128, **kw)

  # -- axes and shapes ------------------------------------------------------
  @functools.cached_property
  def nodal_axes(self):
    lon = np.linspace(0, 2 * np.pi, self.longitude_nodes, endpoint=False)
    sin_lat, _ = LATITUDE_SPACINGS[self.latitude_spacing](self.latitude_nodes)
    return lon, sin_lat

  @property
  def nodal_shape(self):
    return (self.longitude_nodes, self.latitude_nodes)

  @functools.cached_property
  def modal_axes(self):
    m_pos = np.arange(1, self.longitude_wavenumbers)
    m_pos_neg = np.stack([m_pos, -m_pos], axis=1).ravel()
    return (np.concatenate([[0], m_pos_neg]).astype(int),
            np.arange(self.total_wavenumbers))

  @property
  def modal_shape(self):
    return (2 * self.longitude_wavenumbers - 1, self.total_wavenumbers)

  @functools.cached_property
  def modal_mesh(self):
    return np.meshgrid(*self.modal_axes, indexing='ij')

  @functools.cached_property
  def nodal_mesh(self):
    return np.meshgrid(*self.nodal_axes, indexing='ij')

  @functools.cached_property
  def mask(self):
    m, l = self.modal_mesh
    return abs(m) <= l

  @functools.cached_property
  def cos_lat(self):
    return np.sqrt(1 - self.nodal_axes[1] ** 2)

  @functools.cached_property
  def sec2_lat(self):
    return 1 / (1 - self.nodal_axes[1] ** 2)

  @functools.cached_property
  def laplacian_eigenvalues(self):
    l = self.modal_axes[1]
    return -l * (l + 1) / self.radius ** 2

  # -- basis ------------------------------------------------------------
  @functools.cached_property
  def basis(self):
    """(f, p, w) with p rows duplicated for +-m (spherical_harmonic.py:219-260)."""
    f = real_fourier_basis(self.longitude_wavenumbers, self.longitude_nodes)
    wf = 2 * np.pi / self.longitude_nodes
    x, wp = LATITUDE_SPACINGS[self.latitude_spacing](self.latitude_nodes)
    p = legendre_table(self.longitude_wavenumbers, self.total_wavenumbers, x)
    p = np.repeat(p, 2, axis=0)[1:]
    return f, p, wf * wp

  @functools.cached_property
  def _gemm_basis(self):
    """The basis in the compute dtype, laid out for the per-m GEMMs."""
    f, p, w = self.basis
    dt = self.compute_dtype
    if dt != np.float64:
      # XLA's CPU backend flushes subnormals to zero; the Legendre values
      # near the poles at large m would otherwise be subnormal in float32
      # and slow every product that touches them.
      p = np.where(np.abs(p) < np.finfo(dt).tiny, 0.0, p)
    return (np.ascontiguousarray(f, dt), np.ascontiguousarray(f.T, dt),
            np.ascontiguousarray(p, dt),
            np.ascontiguousarray(np.swapaxes(p, -1, -2), dt), w.astype(dt))

  # -- transforms -------------------------------------------------------
  # The reference contracts with einsum over all leading (field) axes at
  # once, which XLA lowers to one GEMM per m with the fields as the GEMM's N
  # dimension.  The same shape here: fields are moved to the last axis, so
  # each contraction is a batched matmul over m of (J x L) @ (L x F) and the
  # Fourier sums one (I x M) @ (M x J F) product.
  def to_nodal(self, x):
    """Inverse transform (spherical_harmonic.py:262-269)."""
    f, _, p, _, _ = self._gemm_basis
    x = np.asarray(x, dtype=self.compute_dtype)
    lead = x.shape[:-2]
    m_, l_ = x.shape[-2:]
    xf = x.reshape((-1, m_, l_)).transpose(1, 2, 0)          # (M, L, F)
    px = np.matmul(p, xf)                                    # 'mjl,...ml->...mj'
    if self.compute_dtype != np.float64:
      px[np.abs(px) < np.finfo(px.dtype).tiny] = 0.0         # flush subnormals
    j_ = px.shape[1]
    z = (f @ px.reshape(m_, -1)).reshape(f.shape[0], j_, -1)  # 'im,...mj->...ij'
    return np.moveaxis(z, -1, 0).reshape(lead + z.shape[:2])

  def to_modal(self, z):
    """Forward transform (spherical_harmonic.py:271-280)."""
    _, ft, _, pt, w = self._gemm_basis
    z = np.asarray(z, dtype=self.compute_dtype)
    lead = z.shape[:-2]
    i_, j_ = z.shape[-2:]
    zf = (w * z).reshape((-1, i_, j_)).transpose(1, 2, 0)     # (I, J, F)
    fwx = (ft @ zf.reshape(i_, -1)).reshape(ft.shape[0], j_, -1)  # 'im,...ij->...mj'
    out = np.matmul(pt, fwx)                                 # 'mjl,...mj->...ml'
    return np.moveaxis(out, -1, 0).reshape(lead + out.shape[:2])

  # -- operators --------------------------------------------------------
  def laplacian(self, x):
    """spherical_harmonic.py:1033-1036."""
    return x * self.laplacian_eigenvalues

  def inverse_laplacian(self, x):
    """spherical_harmonic.py:1038-1046."""
    with np.errstate(divide='ignore', invalid='ignore'):
      inv = 1 / self.laplacian_eigenvalues
    inv[0] = 0
    return x * inv

  def clip_wavenumbers(self, x, n: int = 1):
    """Zero the highest n total wavenumbers (spherical_harmonic.py:1048-1061)."""
    if n <= 0:
      raise ValueError(f'`n` must be >= 0; got {n}.')
    mask = np.ones(self.total_wavenumbers)
    mask[-n:] = 0
    return x * mask

  @functools.cached_property
  def _derivative_recurrence_weights(self):
    """spherical_harmonic.py:1063-1070."""
    m, l = self.modal_mesh
    a = np.sqrt(self.mask * (l ** 2 - m ** 2) / (4 * l ** 2 - 1))
    a[:, 0] = 0
    b = np.sqrt(self.mask * ((l + 1) ** 2 - m ** 2) / (4 * (l + 1) ** 2 - 1))
    b[:, -1] = 0
    return a, b

  def d_dlon(self, x):
    """spherical_harmonic.py:1072-1077 -> fourier.real_basis_derivative."""
    return real_basis_derivative(x, axis=-2)

  def cos_lat_d_dlat(self, x):
    """spherical_harmonic.py:1079-1093."""
    _, l = self.modal_mesh
    a, b = self._derivative_recurrence_weights
    return (_shift(((l + 1) * a) * x, -1, -1) + _shift((-l * b) * x, +1, -1))

  def sec_lat_d_dlat_cos2(self, x):
    """spherical_harmonic.py:1095-1102."""
    _, l = self.modal_mesh
    a, b = self._derivative_recurrence_weights
    return (_shift(((l - 1) * a) * x, -1, -1)
            + _shift((-(l + 2) * b) * x, +1, -1))

  def cos_lat_grad(self, x, clip: bool = True):
    """spherical_harmonic.py:1104-1111."""
    raw = (self.d_dlon(x) / self.radius, self.cos_lat_d_dlat(x) / self.radius)
    if clip:
      return tuple(self.clip_wavenumbers(r) for r in raw)
    return raw

  @staticmethod
  def k_cross(v):
    """spherical_harmonic.py:1113-1116."""
    return -v[1], v[0]

  def div_cos_lat(self, v, clip: bool = True):
    """spherical_harmonic.py:1118-1128."""
    raw = (self.d_dlon(v[0]) + self.sec_lat_d_dlat_cos2(v[1])) / self.radius
    return self.clip_wavenumbers(raw) if clip else raw

  def curl_cos_lat(self, v, clip: bool = True):
    """spherical_harmonic.py:1130-1140."""
    raw = (self.d_dlon(v[1]) - self.sec_lat_d_dlat_cos2(v[0])) / self.radius
    return self.clip_wavenumbers(raw) if clip else raw

  def integrate(self, z):
    """spherical_harmonic.py:1147-1151."""
    w = self.basis[2] * self.radius ** 2
    return np.einsum('y,...xy->...', w, z)


def get_cos_lat_vector(vorticity, divergence, grid: Grid, clip: bool = True):
  """(u, v) cos(lat) from vorticity/divergence (spherical_harmonic.py:1164-1178)."""
  stream_function = grid.inverse_laplacian(vorticity)
  velocity_potential = grid.inverse_laplacian(divergence)
  a = grid.cos_lat_grad(velocity_potential, clip=clip)
  b = grid.k_cross(grid.cos_lat_grad(stream_function, clip=clip))
  return a[0] + b[0], a[1] + b[1]


def vor_div_to_uv_nodal(grid: Grid, vorticity, divergence, clip: bool = True):
  """spherical_harmonic.py:1197-1210."""
  u, v = get_cos_lat_vector(vorticity, divergence, grid, clip=clip)
  return grid.to_nodal(u) / grid.cos_lat, grid.to_nodal(v) / grid.cos_lat


def uv_nodal_to_vor_div_modal(grid: Grid, u_nodal, v_nodal, clip: bool = True):
  """spherical_harmonic.py:1181-1194."""
  u = grid.to_modal(u_nodal / grid.cos_lat)
  v = grid.to_modal(v_nodal / grid.cos_lat)
  return (grid.curl_cos_lat((u, v), clip=clip),
          grid.div_cos_lat((u, v), clip=clip))


def exponential_filter_scaling(grid: Grid, attenuation=16, order=18,
                               cutoff=0.0) -> np.ndarray:
  """Per-l scaling of filtering.exponential_filter (filtering.py:38-89)."""
  _, total_wavenumber = grid.modal_axes
  k = total_wavenumber / total_wavenumber.max()
  a, c, p = attenuation, cutoff, order
  return np.exp((k > c) * (-a * (((k - c) / (1 - c)) ** (2 * p))))


def horizontal_diffusion_scaling(grid: Grid, scale, order=1) -> np.ndarray:
  """filtering.py:92-100."""
  eigenvalues = grid.laplacian_eigenvalues
  return np.exp(-scale * (-eigenvalues) ** order)


def fast_to_real(x):
  """FastSphericalHarmonics modal rows (m = 0, 0i, 1, -1, 2, -2, ...;
  spherical_harmonic.py:486-497) -> the Real layout (drops the always-zero
  imaginary m = 0 row)."""
  return np.delete(np.asarray(x), 1, axis=-2)


def real_to_fast(x):
  """The Real layout -> FastSphericalHarmonics rows (inserts the zero row)."""
  return np.insert(np.asarray(x), 1, 0.0, axis=-2)
