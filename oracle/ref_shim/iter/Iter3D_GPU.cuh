// Empty stand-in: the host build of the gradient loop needs nothing from it.
#pragma once
