/*
 * Project-written stand-in for the one MKL declaration the reference's
 * sources use outside its MKL wrapper translation unit.  Intel MKL is not
 * installed here; the wrapper (src/ExtLibrary.cpp) is replaced by
 * oracle/ref/ext_library_shim.cpp.  Test infrastructure only.
 */
#ifndef NPME_ORACLE_MKL_SHIM_H
#define NPME_ORACLE_MKL_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif
void mkl_set_num_threads(int nt);
#ifdef __cplusplus
}
#endif
#endif
