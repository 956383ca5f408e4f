// Instantiation unit: REAL=float, operator id 0 (see ieq_common.cuh).
#define IEQ_R float
#define IEQ_OP 0
#include "stage_inst.cuh"
