#ifndef Xyce_N_LAS_Matrix_h
#define Xyce_N_LAS_Matrix_h
#include <vector>
#include <N_LAS_fwd.h>
// CSR value store: row r occupies vals[rowptr[r] .. rowptr[r+1]); operator[](row)
// returns the row's first value so that [row][offset] addresses one entry.
class N_LAS_Matrix {
public:
  N_LAS_Matrix() {}
  N_LAS_Matrix(const std::vector<int> & rowptr) : rowptr_(rowptr), vals_(rowptr.empty() ? 0 : rowptr.back(), 0.0) {}
  N_LAS_Matrix(const std::vector<int> & rowptr, const std::vector<int> & colind)
      : rowptr_(rowptr), colind_(colind), vals_(rowptr.empty() ? 0 : rowptr.back(), 0.0) {}
  double * operator[](int row) { return &vals_[rowptr_[row]]; }
  const double * operator[](int row) const { return &vals_[rowptr_[row]]; }
  void put(double s) { for (auto & x : vals_) x = s; }
  std::vector<double> & values() { return vals_; }
  // Row-edit entry points used only by trivial-stamp helpers; the harness never calls them.
  int getLocalNumRows() const { return rowptr_.empty() ? 0 : (int)rowptr_.size() - 1; }
  bool replaceLocalRow(int, int, double *, int *) { return false; }
  bool putLocalRow(int, int, double *, int *) { return false; }
  std::vector<int> & rowptr() { return rowptr_; }
  // Row views as the reference's matrix offers them (N_LAS_Matrix.h:155, 181): the row's length,
  // its values and its column indices (when the matrix was built with them).
  int getLocalRowLength(int row) const { return rowptr_[row + 1] - rowptr_[row]; }
  int extractLocalRowView(int row, int & n, double *& v, int *& idx) const {
    n = rowptr_[row + 1] - rowptr_[row];
    v = const_cast<double *>(&vals_[rowptr_[row]]);
    idx = colind_.empty() ? 0 : const_cast<int *>(&colind_[rowptr_[row]]);
    return 0;
  }
private:
  std::vector<int> rowptr_, colind_;
  std::vector<double> vals_;
};
#endif
