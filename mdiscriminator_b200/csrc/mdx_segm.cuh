#pragma once
#include "mdx_device.cuh"
