// Configuration header force-included (-include) into every translation unit of the compiled
// reference (oracle build only).  It plays the role of the header pe's CMake build generates
// from cmake/config.h.in: a serial, double-precision build with no MPI, OpenCL, BLAS or viewer.
#ifndef PE_ORACLE_REF_CONFIG_H
#define PE_ORACLE_REF_CONFIG_H
#define PE_MEDIA_PATH
#define PE_OPENCL_KERNEL_PATH
#define PE_PUBLIC
#define PE_PRIVATE
#define PE_PROTECTED
#define PE_NOTHROW
#define HAVE_BLAS 0
#define HAVE_IRRLICHT 0
#define HAVE_MPI 0
#define HAVE_OPENCL 0
#endif
