"""DLPack export of device-resident results (the legacy ``dltensor`` capsule).

The reference hands resident outputs to CuPy / PyTorch as DLPack tensors
(bindings/gbskernels_ext.cpp:209-228).  Here a resident block (or one of its typed
parts) exports a one-dimensional CUDA tensor over its own device memory: no copy.
The capsule's ``DLManagedTensor`` keeps the owning block alive until the consumer
calls the deleter, so a consumer's tensor never outlives the memory; an explicit
``close()`` of the block is deferred until every exported tensor is released.
"""

from __future__ import annotations

import ctypes

_KDL_CUDA = 2
_KDL_INT, _KDL_FLOAT, _KDL_COMPLEX = 0, 2, 5


class _DLDevice(ctypes.Structure):
    _fields_ = [("device_type", ctypes.c_int), ("device_id", ctypes.c_int)]


class _DLDataType(ctypes.Structure):
    _fields_ = [("code", ctypes.c_uint8), ("bits", ctypes.c_uint8), ("lanes", ctypes.c_uint16)]


class _DLTensor(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("device", _DLDevice), ("ndim", ctypes.c_int),
                ("dtype", _DLDataType), ("shape", ctypes.POINTER(ctypes.c_int64)),
                ("strides", ctypes.POINTER(ctypes.c_int64)), ("byte_offset", ctypes.c_uint64)]


class _DLManagedTensor(ctypes.Structure):
    pass


_DELETER = ctypes.CFUNCTYPE(None, ctypes.POINTER(_DLManagedTensor))
_DLManagedTensor._fields_ = [("dl_tensor", _DLTensor), ("manager_ctx", ctypes.c_void_p), ("deleter", _DELETER)]

# live exports: address of the DLManagedTensor -> (struct, shape, owner)
_LIVE: dict[int, tuple] = {}


def _release(addr: int) -> None:
    entry = _LIVE.pop(addr, None)
    if entry is not None:
        entry[2]._export_released()


@_DELETER
def _deleter(mt):
    _release(ctypes.cast(mt, ctypes.c_void_p).value)


_CAPSULE_DESTRUCTOR = ctypes.CFUNCTYPE(None, ctypes.c_void_p)
_PyCapsule_New = ctypes.pythonapi.PyCapsule_New
_PyCapsule_New.restype = ctypes.py_object
_PyCapsule_New.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _CAPSULE_DESTRUCTOR]
_PyCapsule_IsValid = ctypes.pythonapi.PyCapsule_IsValid
_PyCapsule_IsValid.restype = ctypes.c_int
_PyCapsule_IsValid.argtypes = [ctypes.py_object, ctypes.c_char_p]
_PyCapsule_GetPointer = ctypes.pythonapi.PyCapsule_GetPointer
_PyCapsule_GetPointer.restype = ctypes.c_void_p
_PyCapsule_GetPointer.argtypes = [ctypes.py_object, ctypes.c_char_p]


@_CAPSULE_DESTRUCTOR
def _capsule_destructor(capsule_ptr):
    # an unconsumed capsule (still named "dltensor") releases its tensor itself; a
    # consumer renames it to "used_dltensor" and calls the deleter when done
    cap = ctypes.cast(capsule_ptr, ctypes.py_object)
    if _PyCapsule_IsValid(cap, b"dltensor"):
        _release(_PyCapsule_GetPointer(cap, b"dltensor"))


_DTYPES = {"<c16": (_KDL_COMPLEX, 128), "<f8": (_KDL_FLOAT, 64), "<i4": (_KDL_INT, 32)}


def capsule(owner, data_addr: int, n: int, typestr: str, device_id: int):
    """A ``dltensor`` capsule over n elements at data_addr (device memory of `owner`)."""
    code, bits = _DTYPES[typestr]
    shape = (ctypes.c_int64 * 1)(n)
    mt = _DLManagedTensor()
    mt.dl_tensor.data = ctypes.c_void_p(data_addr)
    mt.dl_tensor.device = _DLDevice(_KDL_CUDA, device_id)
    mt.dl_tensor.ndim = 1
    mt.dl_tensor.dtype = _DLDataType(code, bits, 1)
    mt.dl_tensor.shape = ctypes.cast(shape, ctypes.POINTER(ctypes.c_int64))
    mt.dl_tensor.strides = ctypes.POINTER(ctypes.c_int64)()  # compact
    mt.dl_tensor.byte_offset = 0
    mt.manager_ctx = None
    mt.deleter = _deleter
    addr = ctypes.addressof(mt)
    _LIVE[addr] = (mt, shape, owner)
    owner._export_acquired()
    return _PyCapsule_New(addr, b"dltensor", _capsule_destructor)
