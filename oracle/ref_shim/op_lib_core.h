/* Minimal stand-in for OP2-Common's op_lib_core.h, enough to compile the
 * reference's pyop2/sparsity_utils.cxx unmodified (it reads only these
 * fields, sparsity_utils.cxx:19-26,68-77).  Test infrastructure. */
#ifndef OP_LIB_CORE_SHIM_H
#define OP_LIB_CORE_SHIM_H
#include <stdlib.h>
typedef struct { int size; int exec_size; } op_set_core;
typedef op_set_core *op_set;
typedef struct { op_set from; op_set to; int dim; int *map; } op_map_core;
typedef op_map_core *op_map;
#endif
