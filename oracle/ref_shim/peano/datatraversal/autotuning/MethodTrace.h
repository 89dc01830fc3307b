#pragma once
namespace peano { namespace datatraversal { namespace autotuning {
enum class MethodTrace { UserDefined0, UserDefined1, UserDefined2, UserDefined3, UserDefined4,
  UserDefined5, UserDefined6, UserDefined7, UserDefined8, UserDefined9, UserDefined10, UserDefined11,
  UserDefined12, UserDefined13, UserDefined14, UserDefined15, UserDefined16, UserDefined17,
  UserDefined18, UserDefined19, UserDefined20, UserDefined21, UserDefined22, UserDefined23,
  UserDefined24, UserDefined25, UserDefined26, UserDefined27, UserDefined28, UserDefined29 };
}}}
