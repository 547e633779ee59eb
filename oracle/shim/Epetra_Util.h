#ifndef SHIM_EPETRA_UTIL_H
#define SHIM_EPETRA_UTIL_H
class Epetra_Util {
public:
  Epetra_Util() : seed_(12345u) {}
  double RandomDouble() { seed_ = seed_ * 1103515245u + 12345u; return 2.0 * ((seed_ >> 1) / 2147483648.0) - 1.0; }
  int SetSeed(unsigned int s) { seed_ = s; return 0; }
  unsigned int Seed() const { return seed_; }
private:
  unsigned int seed_;
};
#endif
