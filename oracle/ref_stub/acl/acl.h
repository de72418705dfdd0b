/* Stub of the CANN runtime header, just enough for the reference's CPU golden headers
 * (the test golden headers include acl/acl.h through include/cann_ops_blas.h) to compile on a
 * machine without CANN. Test infrastructure only. */
#pragma once
typedef void* aclrtStream;
typedef int aclError;
typedef int aclDataType;
