"""Host/device buffer sets of the CKM1D integrator.

Mirrors ``coupledbubble_control/models/buffers.py`` (buffer dataclasses
:29-71, BufferOps :74-200): the same groups, field names, shapes and in-place
semantics.  Device arrays are ``torch`` CUDA tensors instead of cupy/numba
arrays; the B200 library only ever sees their raw device pointers.

Shapes (reference ``models/model.py:56-106``):
  actual_time/time_end/time_begin/time_step  (NS,)            float64
  actual_state                              (SD, NS, TILE)    float64
  unit_params                               (NUP, NS, TILE)   float64
  system_params                             (NSP, NS)         float64
  control_params                            (NCP, NS)         float64
  coupling_matrices                         (NCM, UPS, NS, TILE) float64
  dense_index                               (NS,)             int32
  dense_time                                (NDO, NS)         float64
  dense_state                               (NDO, SD, NS, TILE) float64
  actual_event                              (NS,)             float64
  status_flags + four counters              (NS,)             int32
"""
from __future__ import annotations

from dataclasses import dataclass, fields
from typing import Any, Tuple

import numpy as np


@dataclass(slots=True)
class Buffer:
    pass


@dataclass(slots=True)
class ActualStateBuffer(Buffer):
    actual_time: Any
    time_end: Any
    time_begin: Any
    time_step: Any
    actual_state: Any


@dataclass(slots=True)
class ParameterBuffer(Buffer):
    unit_params: Any
    system_params: Any
    control_params: Any
    coupling_matrices: Any


@dataclass(slots=True)
class DenseOutputBuffer(Buffer):
    dense_index: Any
    dense_time: Any
    dense_state: Any


@dataclass(slots=True)
class StatusBuffer:
    actual_event: Any
    status_flags: Any
    total_steps: Any
    rejected_steps: Any
    convergece_success: Any        # (sic) field name of the reference
    convergence_failures: Any


@dataclass(slots=True)
class BufferSet:
    state: ActualStateBuffer
    params: ParameterBuffer
    dense: DenseOutputBuffer
    status: StatusBuffer


class BufferOps:
    """Creates device copies of host buffers and copies between them.

    ``backend`` None keeps numpy arrays (the reference's host-only mode);
    ``BackendName.B200`` creates torch CUDA tensors.
    """

    def __init__(self, backend=None, device: str = "cuda") -> None:
        self.backend = backend
        self.device = device

    def _on_device(self) -> bool:
        from ..backends import BackendName
        return self.backend == BackendName.B200

    def from_host_ary(self, src, *, stream=None):
        host = np.ascontiguousarray(src)
        if self._on_device():
            import torch
            t = torch.from_numpy(host).to(self.device, non_blocking=False)
            return t.contiguous()
        return host.copy()

    def create_device_state(self, src_buf, stream=None):
        return ActualStateBuffer(**{f.name: self.from_host_ary(getattr(src_buf, f.name))
                                    for f in fields(src_buf)})

    def create_device_params(self, src_buf, stream=None):
        return ParameterBuffer(**{f.name: self.from_host_ary(getattr(src_buf, f.name))
                                  for f in fields(src_buf)})

    def create_device_dense_output(self, src_buf, stream=None):
        return DenseOutputBuffer(**{f.name: self.from_host_ary(getattr(src_buf, f.name))
                                    for f in fields(src_buf)})

    def create_device_status(self, src_buf, stream=None):
        return StatusBuffer(**{f.name: self.from_host_ary(getattr(src_buf, f.name))
                               for f in fields(src_buf)})

    def sync_to_device(self, src_buf, dst_buf, stream=None):
        """Host -> device copy between existing buffers (in place)."""
        for f in fields(src_buf):
            self._copy_h2d(getattr(src_buf, f.name), getattr(dst_buf, f.name))

    def sync_to_host(self, src_buf, dst_buf, stream=None):
        """Device -> host copy between existing buffers (in place)."""
        for f in fields(src_buf):
            self._copy_d2h(getattr(src_buf, f.name), getattr(dst_buf, f.name))

    def _copy_h2d(self, src, dst):
        if self._on_device():
            import torch
            dst.copy_(torch.from_numpy(np.ascontiguousarray(src)))
        else:
            np.copyto(dst, src)

    def _copy_d2h(self, src, dst):
        if self._on_device():
            np.copyto(dst, src.cpu().numpy())
        else:
            np.copyto(dst, src)


def shape_of(x) -> Tuple[int, ...]:
    return tuple(x.shape)


def data_ptr(x) -> int:
    """Raw address of a torch tensor or numpy array (0 for None)."""
    if x is None:
        return 0
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    return int(x.ctypes.data)
