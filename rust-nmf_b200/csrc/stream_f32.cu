// stream_f32.cu -- the TMA streaming passes with an f32 V (FP32 form).
#define STREAM_T float
#define STREAM_FACTORY stream_ops_f32
#include "stream_inst.cuh"
