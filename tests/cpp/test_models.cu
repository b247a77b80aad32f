// The models in the generated form (model_test_ar1.cuh,
// model_l96_generated.cuh) compiled into a shared library that hands their
// bpf_model_ops tables to a caller (the Python tests, through ctypes, pass
// them to bpf_create_model).  Built twice: -DBPF_REAL=double and
// -DBPF_REAL=float, both with -fmad=false (expression order of the model
// source).
#include "bpf_model.cuh"
#include "model_test_ar1.cuh"
#include "model_l96_generated.cuh"

extern "C" bpf_model_ops test_ar1_ops(void) { return bpf::model_ops<test_ar1::ModelTest>(); }
extern "C" bpf_model_ops test_l96_ops(void) { return bpf::model_ops<l96_gen::ModelL96>(); }
