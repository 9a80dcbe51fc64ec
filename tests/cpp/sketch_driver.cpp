// A driver with the reference's call pattern (driver/main.cpp:42-77 main_driver,
// :79-141 dense_driver / sparse_driver, :143-210 main), compiled against the
// C++ drop-in layer include/skema.hpp and linked with libskema_b200.so. Only
// the sketch solver exists here; the other solvers print a notice.
#include <chrono>
#include <iostream>
#include <string>

#include "skema.hpp"

template <typename MatrixType>
int main_driver(const MatrixType& matrix, const Skema::AlgParams& algParams) {
  std::cout << "\nMatrix: " << algParams.matrix_m << " x " << algParams.matrix_n << std::endl;
  std::cout << "Solver: " << Skema::Solver_Method::names[algParams.solver] << std::endl;
  switch (Skema::Solver_Method::types[algParams.solver]) {
    case Skema::Solver_Method::SKETCH: {
      auto [U, S, V] = Skema::sketchysvd(matrix, algParams);
      std::cout << "svals:";
      for (size_type i = 0; i < S.extent(0); ++i) std::cout << " " << S(i);
      std::cout << std::endl;
      break;
    }
    default:
      std::cout << "only the sketch solver is provided" << std::endl;
      return 2;
  }
  return 0;
}

int dense_driver(const std::filesystem::path& inputfilename, Skema::AlgParams& algParams) {
  matrix_type matrix = Skema::read_matrix<matrix_type>(inputfilename);
  algParams.matrix_m = matrix.extent(0);
  algParams.matrix_n = matrix.extent(1);
  if (algParams.kernel_func != Skema::Kernel_Map::NONE) {  // rows of the file are the kernel's points
    algParams.matrix_n = algParams.matrix_m;
    algParams.issymmetric = !algParams.force_three_sketch;
  }
  algParams.matrix_nnz = algParams.matrix_m * algParams.matrix_n;
  algParams.issparse = false;
  return main_driver(matrix, algParams);
}

int sparse_driver(const std::filesystem::path& inputfilename, Skema::AlgParams& algParams) {
  crs_matrix_type matrix = Skema::read_matrix<crs_matrix_type>(inputfilename);
  algParams.matrix_m = matrix.numRows();
  algParams.matrix_n = matrix.numCols();
  algParams.matrix_nnz = matrix.nnz();
  algParams.issparse = true;
  return main_driver(matrix, algParams);
}

int main(int argc, char* argv[]) {
  auto args = Skema::build_arg_list(argc, argv);
  const bool help = Skema::parse_bool(args, "--help", "--no-help", false);
  if (argc < 2 || help) {
    Skema::AlgParams::print_help(std::cout);
    return 0;
  }
  Skema::AlgParams algParams;
  std::filesystem::path inputfilename = Skema::parse_filepath(args, "--input", "");
  if (inputfilename.empty()) {
    std::cout << "Must provide matrix input" << std::endl;
    return 1;
  }
  algParams.parse(args);
  if (Skema::check_and_print_unused_args(args, std::cout)) return 1;
  if (algParams.print_level > 0) algParams.print(std::cout);
  return algParams.issparse ? sparse_driver(inputfilename, algParams) : dense_driver(inputfilename, algParams);
}
