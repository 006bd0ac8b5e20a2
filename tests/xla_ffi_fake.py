"""A stand-in for XLA's side of the FFI C ABI (test helper).

jaxlib is not installable here, so the tests play XLA: they build the call
frame XLA would pass (xla/ffi/api/c_api.h, API version 0.1: buffers, scalar
attributes, the metadata extension) with ctypes, provide the two API
functions the handlers call (error creation, stream lookup) and call the
handler symbols of librrtmg_b200.so directly."""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_int, c_int64, c_size_t, c_uint32, c_void_p

F32, F64, S32, U8 = 11, 12, 4, 6
STAGE_EXECUTE = 3
INVALID_ARGUMENT, UNIMPLEMENTED, INTERNAL = 3, 12, 13


class ExtBase(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("type", c_int), ("next", c_void_p)]


class ApiVersion(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("major_version", c_int),
                ("minor_version", c_int)]


class ErrorCreateArgs(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("message", c_char_p), ("errc", c_int)]


class StreamGetArgs(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("ctx", c_void_p), ("stream", c_void_p)]


ERROR_CREATE = ctypes.CFUNCTYPE(c_void_p, POINTER(ErrorCreateArgs))
STREAM_GET = ctypes.CFUNCTYPE(c_void_p, POINTER(StreamGetArgs))


class Api(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("api_version", ApiVersion),
                ("internal_api", c_void_p), ("error_create", ERROR_CREATE), ("error_get_message", c_void_p),
                ("error_destroy", c_void_p), ("handler_register", c_void_p), ("stream_get", STREAM_GET)]


class Buffer(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("dtype", c_int), ("data", c_void_p),
                ("rank", c_int64), ("dims", POINTER(c_int64))]


class Args(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("size", c_int64),
                ("types", POINTER(c_int)), ("args", POINTER(c_void_p))]


class ByteSpan(ctypes.Structure):
    _fields_ = [("ptr", c_char_p), ("len", c_size_t)]


class Scalar(ctypes.Structure):
    _fields_ = [("dtype", c_int), ("value", c_void_p)]


class Attrs(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("size", c_int64),
                ("types", POINTER(c_int)), ("names", POINTER(POINTER(ByteSpan))), ("attrs", POINTER(c_void_p))]


class CallFrame(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("api", POINTER(Api)), ("ctx", c_void_p),
                ("stage", c_int), ("args", Args), ("rets", Args), ("attrs", Attrs)]


class Metadata(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("api_version", ApiVersion), ("traits", c_uint32)]


class MetadataExt(ctypes.Structure):
    _fields_ = [("extension_base", ExtBase), ("metadata", POINTER(Metadata))]


class FakeXla:
    """Builds call frames and records the errors a handler creates."""

    def __init__(self, stream: int = 0):
        self.errors = []          # (code, message) per XLA_FFI_Error_Create call
        self.stream = stream
        self._keep = []
        self._error_cells = []

        def error_create(args):
            a = args.contents
            self.errors.append((a.errc, a.message.decode()))
            cell = ctypes.c_int(len(self.errors))   # an opaque non-null XLA_FFI_Error*
            self._error_cells.append(cell)
            return ctypes.addressof(cell)

        def stream_get(args):
            args.contents.stream = self.stream
            return None

        self._error_create = ERROR_CREATE(error_create)
        self._stream_get = STREAM_GET(stream_get)
        self.api = Api(struct_size=ctypes.sizeof(Api), error_create=self._error_create,
                       stream_get=self._stream_get)
        self.api.api_version = ApiVersion(struct_size=ctypes.sizeof(ApiVersion), major_version=0, minor_version=1)

    def _buffer(self, dtype, ptr, shape):
        dims = (c_int64 * len(shape))(*shape)
        b = Buffer(struct_size=ctypes.sizeof(Buffer), dtype=dtype, data=ptr, rank=len(shape), dims=dims)
        self._keep += [dims, b]
        return ctypes.addressof(b)

    def frame(self, operands, results, attrs: dict, stage: int = STAGE_EXECUTE) -> CallFrame:
        """operands / results: lists of (dtype, data pointer, shape); attrs: name ->
        (dtype, value)."""
        def seq(items):
            n = len(items)
            types = (c_int * n)(*([1] * n))
            ptrs = (c_void_p * n)(*[self._buffer(*it) for it in items])
            self._keep += [types, ptrs]
            return Args(struct_size=ctypes.sizeof(Args), size=n, types=types, args=ptrs)

        names = sorted(attrs)  # XLA passes attributes sorted by name
        n = len(names)
        spans, scalars = [], []
        for name in names:
            dtype, value = attrs[name]
            ctype = {F32: ctypes.c_float, F64: ctypes.c_double, S32: ctypes.c_int32}[dtype]
            cell = ctype(value)
            sc = Scalar(dtype=dtype, value=ctypes.addressof(cell))
            span = ByteSpan(ptr=name.encode(), len=len(name))
            self._keep += [cell, sc, span]
            spans.append(ctypes.pointer(span))
            scalars.append(ctypes.addressof(sc))
        at = Attrs(struct_size=ctypes.sizeof(Attrs), size=n, types=(c_int * n)(*([3] * n)),
                   names=(POINTER(ByteSpan) * n)(*spans), attrs=(c_void_p * n)(*scalars))
        self._keep.append(at)
        f = CallFrame(struct_size=ctypes.sizeof(CallFrame), api=ctypes.pointer(self.api), ctx=None, stage=stage,
                      args=seq(operands), rets=seq(results), attrs=at)
        self._keep.append(f)
        return f

    def metadata_frame(self):
        md = Metadata(struct_size=ctypes.sizeof(Metadata))
        ext = MetadataExt(extension_base=ExtBase(struct_size=ctypes.sizeof(MetadataExt), type=1, next=None),
                          metadata=ctypes.pointer(md))
        f = CallFrame(struct_size=ctypes.sizeof(CallFrame), api=ctypes.pointer(self.api),
                      extension_start=ctypes.addressof(ext), stage=0)
        self._keep += [md, ext, f]
        return f, md


def handler(lib, name: str):
    fn = getattr(lib, name)
    fn.restype = c_void_p
    fn.argtypes = [POINTER(CallFrame)]
    return fn
