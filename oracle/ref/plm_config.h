/* Stand-in for Plastimatch's cmake-generated plm_config.h, used only when
 * the reference's B-spline cost-function sources are compiled as a test
 * oracle (see ../build_ref.sh).  Values describe a 64-bit Linux build with
 * OpenMP and without CUDA, ITK, DCMTK or any other optional library. */
#ifndef __plm_config_h__
#define __plm_config_h__
#define MACHINE_IS_64_BIT 1
#define UNIX 1
#define HAVE_NULLPTR 1
#define HAVE_SYS_STAT_H 1
#define HAVE_STDINT_H 1
#define OPENMP_FOUND 1
#define SHARED_PTR_USE_MEMORY 1
#define CMAKE_SIZEOF_UINT 4
#define CMAKE_SIZEOF_ULONG 8
#define CMAKE_SIZEOF_ULONGLONG 8
#define CMAKE_SIZEOF_SIZE_T 8
#define PLM_BIG_ENDIAN 0
#define libLBFGS_FOUND 1
#ifdef __cplusplus
#define EXTERNC extern "C"
#else
#define EXTERNC
#endif
#endif
