// Instantiation unit: REAL=float, operator id 1 (see ieq_common.cuh).
#define IEQ_R float
#define IEQ_OP 1
#include "stage_inst.cuh"
