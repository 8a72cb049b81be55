"""``Field``: a 3-component grid field held in one flat device tensor.

Same storage contract as upstream ``wakis.Field`` (wakis/field.py:19-348):
``array`` has length 3N = 3*Nx*Ny*Nz and holds the x, y and z blocks; inside a
block the flat index is n = i + j*Nx + k*Nx*Ny (Fortran order).  The data
live in a ``torch.Tensor`` (CUDA when a GPU is used); ``toarray()`` returns
that tensor, indexing with ``field[i, j, k, 'x'|'y'|'z'|'Abs']`` returns a
host numpy copy (as upstream's GPU path does with ``.get()``), assignment
accepts numpy arrays, scalars or tensors.
"""

import numpy as np
import torch

_COMP = {0: 0, 1: 1, 2: 2, "x": 0, "y": 1, "z": 2}

_TORCH_DTYPE = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
                np.dtype(np.int8): torch.int8, np.dtype(np.complex128): torch.complex128}


def torch_dtype(dtype):
    return _TORCH_DTYPE[np.dtype(dtype)]


def default_device(use_gpu=True):
    if use_gpu and torch.cuda.is_available():
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


class Field:
    """3-vector field on an (Nx, Ny, Nz) grid backed by a flat torch tensor."""

    xp = torch   # array module of the storage (upstream: numpy or cupy)

    def __init__(self, Nx, Ny, Nz, dtype=float, use_ones=False, use_gpu=True, device=None,
                 array=None):
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.N = self.Nx * self.Ny * self.Nz
        self.dtype = np.dtype(dtype).type
        self.device = torch.device(device) if device is not None else default_device(use_gpu)
        self.on_gpu = self.device.type == "cuda"
        if array is not None:
            self._array = array
        else:
            fill = torch.ones if use_ones else torch.zeros
            self._array = fill(3 * self.N, dtype=torch_dtype(self.dtype), device=self.device)

    # ------------------------------------------------------------------ data
    @property
    def array(self):
        return self._array

    @array.setter
    def array(self, value):
        self.fromarray(value)

    def toarray(self):
        """The flat (3N,) tensor (live storage, not a copy)."""
        return self.array

    def fromarray(self, array):
        """Copy a flat (3N,) array (numpy or torch) into the field."""
        self._before_write()
        self.array.copy_(self._as_tensor(array).reshape(-1))

    def numpy(self):
        """Host copy of the flat array."""
        return self.array.detach().cpu().numpy()

    def get(self):
        return self.numpy()

    def _as_tensor(self, value):
        if isinstance(value, torch.Tensor):
            return value.to(device=self.device, dtype=self.array.dtype)
        return torch.as_tensor(np.asarray(value), device=self.device).to(self.array.dtype)

    def _before_write(self):
        """Hook for owners that must act before the field changes."""

    # ------------------------------------------------------------- matrices
    def _comp(self, key):
        if key not in _COMP:
            raise IndexError("Component id not valid")
        d = _COMP[key]
        flat = self.array[d * self.N:(d + 1) * self.N]
        # Fortran (i fastest) view indexed [i, j, k]
        return flat.view(self.Nz, self.Ny, self.Nx).permute(2, 1, 0)

    def to_matrix(self, key):
        """(Nx, Ny, Nz) view of one component (indexed [i, j, k])."""
        return self._comp(key)

    def from_matrix(self, mat, key):
        self._before_write()
        self._comp(key).copy_(self._as_tensor(mat).reshape(self.Nx, self.Ny, self.Nz))

    @property
    def field_x(self):
        return self.array[0:self.N]

    @field_x.setter
    def field_x(self, value):
        self._set_block(0, value)

    @property
    def field_y(self):
        return self.array[self.N:2 * self.N]

    @field_y.setter
    def field_y(self, value):
        self._set_block(1, value)

    @property
    def field_z(self):
        return self.array[2 * self.N:3 * self.N]

    @field_z.setter
    def field_z(self, value):
        self._set_block(2, value)

    def _set_block(self, d, value):
        """Component d from an (Nx, Ny, Nz) matrix or a flat N array
        (upstream field_x/field_y/field_z setters, wakis/field.py:95-120)."""
        if np.ndim(value) > 1:
            self.from_matrix(value, d)
        else:
            self._before_write()
            self.array[d * self.N:(d + 1) * self.N] = self._as_tensor(value).reshape(-1)

    def get_abs(self, as_matrix=True):
        """|F| as an (Nx, Ny, Nz) host array, or flat (N,) with
        as_matrix=False (upstream get_abs, wakis/field.py:536-574)."""
        if as_matrix:
            x, y, z = (self._comp(k).detach().cpu().numpy() for k in "xyz")
        else:
            x, y, z = (v.detach().cpu().numpy() for v in (self.field_x, self.field_y,
                                                          self.field_z))
        # on the host with numpy's correctly rounded square root, as upstream
        return np.sqrt(x ** 2 + y ** 2 + z ** 2)

    def compute_ijk(self, n):
        """(i, j, k) of the lexicographic index n (upstream compute_ijk,
        wakis/field.py:511-534)."""
        if n > self.N:
            raise IndexError("Lexico-graphic index cannot be higher than product of dimensions")
        k = n // (self.Nx * self.Ny)
        i = (n - k * self.Nx * self.Ny) % self.Nx
        j = (n - k * self.Nx * self.Ny) // self.Nx
        return i, j, k

    # -------------------------------------------------------------- indexing
    def __getitem__(self, key):
        if isinstance(key, tuple):
            if len(key) != 4:
                raise IndexError("Need 3 indexes and component to access the field")
            if isinstance(key[3], str) and key[3].lower() == "abs":
                return self.get_abs()[key[0], key[1], key[2]]
            v = self._comp(key[3])[key[0], key[1], key[2]]
            out = v.detach().cpu().numpy()
            return out if out.ndim else out[()]
        if isinstance(key, (int, np.integer)):
            if key <= self.N:
                return self.array[int(key)].item()
            raise IndexError("Lexico-graphic index cannot be higher than product of dimensions")
        if isinstance(key, slice):
            return self.array[key].detach().cpu().numpy()
        raise ValueError("key must be a 3-tuple or an integer")

    def __setitem__(self, key, value):
        self._before_write()
        if isinstance(key, tuple):
            if len(key) != 4:
                raise IndexError("Need 3 indexes and component to access the field")
            view = self._comp(key[3])[key[0], key[1], key[2]]
            if isinstance(view, torch.Tensor) and view.dim() > 0:
                view.copy_(self._as_tensor(value).reshape(view.shape) if np.ndim(value)
                           else self._as_tensor(value).expand(view.shape))
            else:
                self._comp(key[3])[key[0], key[1], key[2]] = self._as_tensor(value)
        elif isinstance(key, (int, np.integer)):
            if key <= self.N:
                self.array[int(key)] = self._as_tensor(value)
            else:
                raise IndexError(
                    "Lexico-graphic index cannot be higher than product of dimensions")
        elif isinstance(key, slice):
            self.array[key] = self._as_tensor(value)
        else:
            raise IndexError("key must be a 3-tuple or an integer")

    # ------------------------------------------------------------ arithmetic
    def _new(self, array):
        return Field(self.Nx, self.Ny, self.Nz, dtype=self.dtype, device=self.device,
                     array=array.to(torch_dtype(self.dtype)))

    def _operand(self, other):
        if isinstance(other, Field):
            return other.array
        if np.isscalar(other):
            return other
        t = self._as_tensor(other)
        if t.dim() > 1:   # (Nx, Ny, Nz) matrix applied to every component
            t = t.permute(2, 1, 0).reshape(-1).repeat(3)
        return t

    def __mul__(self, other):
        return self._new(self.array * self._operand(other))

    __rmul__ = __mul__

    def __add__(self, other):
        return self._new(self.array + self._operand(other))

    __radd__ = __add__

    def __truediv__(self, other):
        return self._new(self.array / self._operand(other))

    def copy(self):
        return self._new(self.array.clone())

    def to_gpu(self):
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device")
        self._array = self._array.cuda()
        self.device = self._array.device
        self.on_gpu = True

    def from_gpu(self):
        self._array = self._array.cpu()
        self.device = self._array.device
        self.on_gpu = False

    def __repr__(self):
        return f"Field({self.Nx}x{self.Ny}x{self.Nz}, {np.dtype(self.dtype).name}, {self.device})"


class StateField(Field):
    """Field whose storage alternates between two buffers.

    The fused step kernel reads one buffer and writes the other; ``owner``
    holds the parity, so ``array`` always returns the live buffer.  Writes
    go through ``fromarray``, ``from_matrix`` or item assignment, which tell
    the owner first (it keeps J = sigma*E and the state of the PEC faces in
    step with E); an in-place change of the tensor ``array`` returns is not
    seen by the solver.
    """

    def __init__(self, owner, bufs, Nx, Ny, Nz, dtype):
        self._owner = owner
        self._bufs = bufs
        super().__init__(Nx, Ny, Nz, dtype=dtype, device=bufs[0].device, array=bufs[0])

    @property
    def array(self):
        return self._bufs[self._owner._par]

    @array.setter
    def array(self, value):
        self.fromarray(value)

    def _before_write(self):
        self._owner._field_written(self)
