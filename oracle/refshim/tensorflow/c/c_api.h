/* Test infrastructure only: a declaration-compatible stand-in for the 15 TensorFlow C-API
 * entry points that the reference's pair_nnp.cpp calls (pair_nnp.cpp:12-119). It declares
 * opaque types and prototypes; tf_shim.cpp implements them with a CPU network so that the
 * reference's NNPOTENTIAL_TBL descriptor and back-projection code can run as the oracle.
 * No TensorFlow code is contained or needed. */
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>

extern "C" {

typedef enum TF_DataType { TF_FLOAT = 1, TF_DOUBLE = 2, TF_INT32 = 3 } TF_DataType;
typedef enum TF_Code { TF_OK = 0, TF_UNKNOWN = 2, TF_INVALID_ARGUMENT = 3 } TF_Code;

typedef struct TF_Graph TF_Graph;
typedef struct TF_Status TF_Status;
typedef struct TF_SessionOptions TF_SessionOptions;
typedef struct TF_Session TF_Session;
typedef struct TF_Operation TF_Operation;
typedef struct TF_Tensor TF_Tensor;
typedef struct TF_Buffer TF_Buffer;
typedef struct TF_Output { TF_Operation* oper; int index; } TF_Output;

TF_Graph* TF_NewGraph(void);
void TF_DeleteGraph(TF_Graph*);
TF_Status* TF_NewStatus(void);
void TF_DeleteStatus(TF_Status*);
TF_Code TF_GetCode(const TF_Status*);
const char* TF_Message(const TF_Status*);
TF_SessionOptions* TF_NewSessionOptions(void);
void TF_DeleteSessionOptions(TF_SessionOptions*);
void TF_SetConfig(TF_SessionOptions*, const void* proto, size_t proto_len, TF_Status*);
TF_Session* TF_LoadSessionFromSavedModel(const TF_SessionOptions*, const TF_Buffer* run_options,
                                         const char* export_dir, const char* const* tags, int ntags,
                                         TF_Graph* graph, TF_Buffer* meta_graph_def, TF_Status*);
TF_Operation* TF_GraphOperationByName(TF_Graph*, const char* oper_name);
TF_Tensor* TF_AllocateTensor(TF_DataType, const int64_t* dims, int num_dims, size_t len);
void* TF_TensorData(const TF_Tensor*);
void TF_DeleteTensor(TF_Tensor*);
void TF_SessionRun(TF_Session* session, const TF_Buffer* run_options,
                   const TF_Output* inputs, TF_Tensor* const* input_values, int ninputs,
                   const TF_Output* outputs, TF_Tensor** output_values, int noutputs,
                   const TF_Operation* const* target_opers, int ntargets,
                   TF_Buffer* run_metadata, TF_Status*);
}
