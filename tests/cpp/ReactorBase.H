// Test stand-in for the parts of AMReX and PelePhysics' ReactorBase that the
// ReactorB200 shim uses (types and signatures as the call sites in
// Source/PeleLMeX_Setup.cpp:146-155 and Source/PeleLMeX_Reactions.cpp:101-108
// use them).  Only for compiling and exercising the shim on the host.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

namespace amrex {
using Real = double;
using gpuStream_t = void*;

struct Dim3 {
  int x, y, z;
  int operator[](int d) const { return d == 0 ? x : (d == 1 ? y : z); }
};

template <class T>
struct Array4 {
  T* p = nullptr;
  long long jstride = 0, kstride = 0, nstride = 0;
  Dim3 begin{0, 0, 0}, end{1, 1, 1};
  int ncomp = 1;
  T& operator()(int i, int j, int k, int n = 0) const {
    return p[(i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride + n * nstride];
  }
};

struct Box {
  int lo[3], hi[3];
  int smallEnd(int d) const { return lo[d]; }
  int bigEnd(int d) const { return hi[d]; }
};

// Input keys "prefix.name" -> value, filled by the host program that
// stands in for the inputs file.
struct ParmParse {
  explicit ParmParse(const std::string& prefix) : prefix_(prefix) {}
  static std::map<std::string, std::string>& table() {
    static std::map<std::string, std::string> t;
    return t;
  }
  template <class T>
  int query(const char* name, T& v) const {
    auto it = table().find(prefix_ + "." + name);
    if (it == table().end()) return 0;
    std::istringstream in(it->second);
    in >> v;
    return 1;
  }
  std::string prefix_;
};

[[noreturn]] inline void Abort(const char* msg) {
  std::fprintf(stderr, "Abort: %s\n", msg);
  std::exit(3);
}
}  // namespace amrex

namespace pele::physics {
struct Fuego {};
struct PhysicsType {
  using eos_type = Fuego;
};
namespace eos {
template <class EosType>
struct EosParm {};
}  // namespace eos
}  // namespace pele::physics

namespace pele::physics::reactions {
// self-registering factory base, in the manner of the one the reference's
// reactors derive from (Register<T> is instantiated once Base is complete)
template <class Base>
struct Factory {
  static std::map<std::string, std::unique_ptr<Base> (*)()>& registry() {
    static std::map<std::string, std::unique_ptr<Base> (*)()> r;
    return r;
  }
  static std::unique_ptr<Base> create(const std::string& name) { return registry().at(name)(); }
  template <class T>
  struct Register : Base {
    static bool add() {
      registry()[T::identifier()] = []() -> std::unique_ptr<Base> { return std::make_unique<T>(); };
      return true;
    }
    static inline bool registered = add();
    Register() { (void)registered; }
  };
};

class ReactorBase : public Factory<ReactorBase> {
public:
  virtual ~ReactorBase() = default;
  virtual int init(int reactor_type, int ncells) = 0;
  virtual void close() = 0;
  virtual void set_typ_vals_ode(const std::vector<amrex::Real>& typ) = 0;
  // Source/PeleLMeX_Setup.cpp:155 passes the EOS parameters after init
  virtual void set_eos_parm(const eos::EosParm<PhysicsType::eos_type>* eos_parm) { m_eos_parm = eos_parm; }
  const eos::EosParm<PhysicsType::eos_type>* m_eos_parm = nullptr;
  virtual int react(const amrex::Box& box, amrex::Array4<amrex::Real> const& rY_in,
                    amrex::Array4<amrex::Real> const& rYsrc_in, amrex::Array4<amrex::Real> const& T_in,
                    amrex::Array4<amrex::Real> const& rEner_in, amrex::Array4<amrex::Real> const& rEner_src_in,
                    amrex::Array4<amrex::Real> const& FC_in, amrex::Array4<int> const& mask,
                    amrex::Real& dt_react, amrex::Real& time, amrex::gpuStream_t stream) = 0;
};
}  // namespace pele::physics::reactions
