// The part of XLA's FFI C ABI (xla/ffi/api/c_api.h, API version 0.1; jaxlib
// ships the header) that the rrtmg custom-call handlers use: the call frame
// XLA passes a handler, its buffers and attributes, the metadata query, and
// the two API functions called (error creation, stream lookup).  Layouts and
// enumerator values are those of the published header, which this image does
// not have; only the fields up to the last one used are declared where XLA
// appends fields to a struct (struct_size tells the versions apart).
#pragma once

#include <cstddef>
#include <cstdint>

extern "C" {

struct XLA_FFI_Error;
struct XLA_FFI_ExecutionContext;
struct XLA_FFI_InternalApi;

enum XLA_FFI_Extension_Type { XLA_FFI_Extension_Metadata = 1 };

struct XLA_FFI_Extension_Base {
  size_t struct_size;
  XLA_FFI_Extension_Type type;
  XLA_FFI_Extension_Base *next;
};

struct XLA_FFI_Api_Version {
  size_t struct_size;
  XLA_FFI_Extension_Base *extension_start;
  int major_version;
  int minor_version;
};

enum XLA_FFI_ExecutionStage {
  XLA_FFI_ExecutionStage_INSTANTIATE = 0,
  XLA_FFI_ExecutionStage_PREPARE = 1,
  XLA_FFI_ExecutionStage_INITIALIZE = 2,
  XLA_FFI_ExecutionStage_EXECUTE = 3,
};

enum XLA_FFI_Error_Code {
  XLA_FFI_Error_Code_OK = 0,
  XLA_FFI_Error_Code_INVALID_ARGUMENT = 3,
  XLA_FFI_Error_Code_RESOURCE_EXHAUSTED = 8,
  XLA_FFI_Error_Code_UNIMPLEMENTED = 12,
  XLA_FFI_Error_Code_INTERNAL = 13,
};

enum XLA_FFI_DataType {
  XLA_FFI_DataType_INVALID = 0,
  XLA_FFI_DataType_S32 = 4,
  XLA_FFI_DataType_S64 = 5,
  XLA_FFI_DataType_U8 = 6,
  XLA_FFI_DataType_F32 = 11,
  XLA_FFI_DataType_F64 = 12,
};

struct XLA_FFI_Error_Create_Args {
  size_t struct_size;
  XLA_FFI_Extension_Base *extension_start;
  const char *message;
  XLA_FFI_Error_Code errc;
};
typedef XLA_FFI_Error *XLA_FFI_Error_Create(XLA_FFI_Error_Create_Args *args);

struct XLA_FFI_Stream_Get_Args {
  size_t struct_size;
  XLA_FFI_Extension_Base *extension_start;
  XLA_FFI_ExecutionContext *ctx;
  void *stream;  // out: the cudaStream_t of the call
};
typedef XLA_FFI_Error *XLA_FFI_Stream_Get(XLA_FFI_Stream_Get_Args *args);

typedef void XLA_FFI_Unused_Fn(void);

struct XLA_FFI_Api {
  size_t struct_size;
  XLA_FFI_Extension_Base *extension_start;
  XLA_FFI_Api_Version api_version;
  XLA_FFI_InternalApi *internal_api;
  XLA_FFI_Error_Create *XLA_FFI_Error_Create;
  XLA_FFI_Unused_Fn *XLA_FFI_Error_GetMessage;
  XLA_FFI_Unused_Fn *XLA_FFI_Error_Destroy;
  XLA_FFI_Unused_Fn *XLA_FFI_Handler_Register;
  XLA_FFI_Stream_Get *XLA_FFI_Stream_Get;
};

struct XLA_FFI_Buffer {
  size_t struct_size;
  XLA_FFI_Extension_Base *extension_start;
  XLA_FFI_DataType dtype;
  void *data;
  int64_t rank;
  int64_t *dims;
};

enum XLA_FFI_ArgType { XLA_FFI_ArgType_BUFFER = 1 };
enum XLA_FFI_RetType { XLA_FFI_RetType_BUFFER = 1 };
enum XLA_FFI_AttrType {
  XLA_FFI_AttrType_ARRAY = 1,
  XLA_FFI_AttrType_DICTIONARY = 2,
  XLA_FFI_AttrType_SCALAR = 3,
  XLA_FFI_AttrType_STRING = 4,
};

struct XLA_FFI_Args {
  size_t struct_size;
  XLA_FFI_Extension_Base *extension_start;
  int64_t size;
  XLA_FFI_ArgType *types;
  void **args;  // XLA_FFI_Buffer* each
};

struct XLA_FFI_Rets {
  size_t struct_size;
  XLA_FFI_Extension_Base *extension_start;
  int64_t size;
  XLA_FFI_RetType *types;
  void **rets;  // XLA_FFI_Buffer* each
};

struct XLA_FFI_ByteSpan {
  const char *ptr;
  size_t len;
};

struct XLA_FFI_Scalar {
  XLA_FFI_DataType dtype;
  void *value;
};

struct XLA_FFI_Attrs {
  size_t struct_size;
  XLA_FFI_Extension_Base *extension_start;
  int64_t size;
  XLA_FFI_AttrType *types;
  XLA_FFI_ByteSpan **names;
  void **attrs;  // XLA_FFI_Scalar* for scalar attributes
};

struct XLA_FFI_CallFrame {
  size_t struct_size;
  XLA_FFI_Extension_Base *extension_start;
  const XLA_FFI_Api *api;
  XLA_FFI_ExecutionContext *ctx;
  XLA_FFI_ExecutionStage stage;
  XLA_FFI_Args args;
  XLA_FFI_Rets rets;
  XLA_FFI_Attrs attrs;
};

typedef uint32_t XLA_FFI_Handler_Traits;

struct XLA_FFI_Metadata {
  size_t struct_size;
  XLA_FFI_Api_Version api_version;
  XLA_FFI_Handler_Traits traits;
};

struct XLA_FFI_Metadata_Extension {
  XLA_FFI_Extension_Base extension_base;
  XLA_FFI_Metadata *metadata;
};

}  // extern "C"
