// stream_f64.cu -- the TMA streaming passes with an f64 V (plain FP64 method).
#define STREAM_T double
#define STREAM_FACTORY stream_ops_f64
#include "stream_inst.cuh"
