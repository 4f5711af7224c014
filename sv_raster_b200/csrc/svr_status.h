/* Status codes shared by the C ABI (include/svr_b200.h) and the kernels. */
#ifndef SVR_STATUS_H_
#define SVR_STATUS_H_

#define SVR_OK 0
#define SVR_ERR_SHAPE 1      /* bad sizes or arguments (reference: AT_ERROR / Python raise) */
#define SVR_ERR_CAPACITY 2   /* an instance or workspace buffer is too small */
#define SVR_ERR_KEYBITS 3    /* sort key would not fit in 64 bits */
#define SVR_ERR_CUDA 4       /* a CUDA runtime call failed */
#define SVR_ERR_DEVICE 5     /* a device-side consistency check tripped (replaces __trap) */
#define SVR_ERR_ALIGN 6      /* a pointer is not aligned as required */

/* Bits of the device error word (written by kernels, read by the host). */
#define SVR_DEVERR_DUP_MISMATCH 0x1u   /* duplicate count != scan difference (forward.cu:565-570) */
#define SVR_DEVERR_RANGE 0x2u          /* tile_last outside its range (backward.cu:122-133) */
#define SVR_DEVERR_CAPACITY 0x4u       /* instances exceeded the caller's capacity */
#define SVR_DEVERR_VOXID 0x8u          /* voxel id does not fit in 29 bits */
#define SVR_DEVERR_LEVEL 0x10u         /* an octree path is deeper than the declared max level */

#endif
