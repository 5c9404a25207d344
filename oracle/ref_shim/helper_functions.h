/* Empty: cuda_shim.h (force-included) declares what the reference uses from this header. */
#pragma once
