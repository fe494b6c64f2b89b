// Device selection (device_t of the reference, src/device/general.h): the
// B200 engine; [device] idx_device picks the CUDA ordinal.
#pragma once

namespace device
{
struct b200_t {};
}
using device_t = device::b200_t;
