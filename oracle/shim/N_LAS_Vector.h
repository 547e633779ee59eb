#ifndef Xyce_N_LAS_Vector_h
#define Xyce_N_LAS_Vector_h
// Oracle shim: the device code only indexes vectors, so a vector here is a dense array that
// either owns its storage or views a caller's buffer (the harness keeps one view per solver
// vector so that devices reading through N_LAS_Vector and through raw pointers see the same data).
#include <vector>
#include <N_LAS_fwd.h>
class N_LAS_Vector {
public:
  explicit N_LAS_Vector(int n = 0) : own_(n, 0.0), p_(own_.data()), n_(n) {}
  N_LAS_Vector(double *view, int n) : p_(view), n_(n) {}
  N_LAS_Vector(const N_LAS_Vector &o) : own_(o.own_), p_(o.own_.empty() ? o.p_ : own_.data()), n_(o.n_) {}
  N_LAS_Vector &operator=(const N_LAS_Vector &o) {
    own_ = o.own_;
    p_ = own_.empty() ? o.p_ : own_.data();
    n_ = o.n_;
    return *this;
  }
  double &operator[](int i) { return p_[i]; }
  const double &operator[](int i) const { return p_[i]; }
  void putScalar(double s) { for (int i = 0; i < n_; ++i) p_[i] = s; }
  int localLength() const { return n_; }
private:
  std::vector<double> own_;
  double *p_;
  int n_;
};
#endif
