#pragma once
// Threads per block of general 1-D kernels in the reference's API.
#define BLOCK_SIZE 256
