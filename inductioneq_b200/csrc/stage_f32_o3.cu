// Instantiation unit: REAL=float, operator id 3 (see ieq_common.cuh).
#define IEQ_R float
#define IEQ_OP 3
#include "stage_inst.cuh"
