// The C++ host side reports a refused C-ABI call as SemError: a database
// with no elements is refused by sem_prepare_mesh before any device call.
// Prints the status; exits 0 when SemError was thrown.
#include <iostream>

#include "prepare_fwd.hpp"

int main() {
  sem_mesh_desc d{};  // nspec = nglob = 0
  try {
    specfwat::Mesh mesh(d);
  } catch (const specfwat::SemError& e) {
    std::cout << e.status() << "\n" << e.what() << "\n";
    return 0;
  }
  return 1;
}
