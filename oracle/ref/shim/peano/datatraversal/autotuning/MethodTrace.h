// stand-in: the grain-size labels are opaque integers here
#pragma once
namespace peano { namespace datatraversal { namespace autotuning {
enum class MethodTrace { UserDefined20, UserDefined21, UserDefined22, UserDefined23, UserDefined24, UserDefined25, UserDefined26 };
}}}
