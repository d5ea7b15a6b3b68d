/* Stand-in for Plastimatch's cmake-generated plm_version.h (oracle build). */
#ifndef __plm_version_h__
#define __plm_version_h__
#define PLASTIMATCH_VERSION_STRING "oracle"
#define PLASTIMATCH_BUILD_NUMBER "oracle"
#endif
