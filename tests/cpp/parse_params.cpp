// Parses its arguments with Skema::AlgParams::parse (include/skema.hpp) and
// prints the sketch fields one per line, "name value", for comparison with
// the Python mirror's parser; a parse error prints "error <message>".
#include <iostream>

#include "skema.hpp"

int main(int argc, char** argv) {
  auto args = Skema::build_arg_list(argc, argv);
  Skema::AlgParams p;
  try {
    p.parse(args);
  } catch (const std::exception& e) {
    std::cout << "error " << e.what() << std::endl;
    return 0;
  }
  std::cout << "matrix_m " << p.matrix_m << "\nmatrix_n " << p.matrix_n << "\nrank " << p.rank << "\nwindow "
            << p.window << "\nsketch_range " << p.sketch_range << "\nsketch_core " << p.sketch_core
            << "\nsketch_eta " << p.sketch_eta << "\nsketch_nu " << p.sketch_nu << "\ndim_redux " << p.dim_redux
            << "\nkernel_func " << p.kernel_func << "\nkernel_gamma " << p.kernel_gamma << "\nsolver " << p.solver
            << "\nissparse " << p.issparse << "\nissymmetric " << p.issymmetric << "\nforce_three_sketch "
            << p.force_three_sketch << "\nprecision " << p.precision << "\nspd_approx " << p.spd_approx
            << "\nseeds";
  for (int s : p.seeds) std::cout << " " << s;
  std::cout << "\nunused";
  for (const auto& a : args) std::cout << " " << a;
  std::cout << std::endl;
  return 0;
}
