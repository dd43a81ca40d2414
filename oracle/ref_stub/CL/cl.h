/*
 * Minimal stand-in for <CL/cl.h>, used ONLY to compile speedynn's CPU
 * backend (speedynn/lib/{nearest_neighbors_feature_selection,util,cpu,
 * loss_functions}.c) as a test oracle.  Those files include gpu.h
 * (speedynn/lib/gpu.h:14), which declares OpenCL-typed globals; with
 * USE_GPU=0 none of them is ever used, so opaque handle types suffice.
 * No OpenCL function is declared or called.
 */
#ifndef SNN_ORACLE_CL_STUB_H
#define SNN_ORACLE_CL_STUB_H

typedef int cl_int;
typedef unsigned int cl_uint;
typedef struct snn_stub_cl_platform_id *cl_platform_id;
typedef struct snn_stub_cl_device_id *cl_device_id;
typedef struct snn_stub_cl_context *cl_context;
typedef struct snn_stub_cl_command_queue *cl_command_queue;
typedef struct snn_stub_cl_mem *cl_mem;
typedef struct snn_stub_cl_program *cl_program;
typedef struct snn_stub_cl_kernel *cl_kernel;
typedef struct snn_stub_cl_event *cl_event;

#endif
