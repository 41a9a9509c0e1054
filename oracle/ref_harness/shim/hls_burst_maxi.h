/* Empty stand-in for the Xilinx hls_burst_maxi.h (unused on the host). */
#pragma once
