#pragma once
// stand-in: nothing from tarch/la/Scalar.h is used by the kernels built here
