// Instantiation unit: REAL=float, operator id 2 (see ieq_common.cuh).
#define IEQ_R float
#define IEQ_OP 2
#include "stage_inst.cuh"
