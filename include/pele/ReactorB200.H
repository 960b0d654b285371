// ReactorB200.H -- the PelePhysics reactor a PeleLMeX build registers to run
// its chemistry advance on the B200 library: peleLM.chem_integrator =
// "ReactorB200" (Source/PeleLMeX_Setup.cpp:149-153) creates it through the
// ReactorBase factory; init / set_typ_vals_ode / react / close are called at
// Source/PeleLMeX_Setup.cpp:146-155, Source/PeleLMeX_Utils.cpp:1472,
// Source/PeleLMeX_Reactions.cpp:101-108 and Source/PeleLMeX.cpp:26.
//
// Header-only; include it in one translation unit of the PelePhysics build
// (Reactions/), link -lb200chem.  The mechanism tables come from
// b200chem_make_mech_desc(), the translation unit that
//   python -m pelelmex_b200.mechgen --mech-desc <mechanism> --out mech_desc.cpp
// writes for the mechanism in use.
//
// Input keys (besides the reference's ode.rtol, ode.atol, cvode.max_order,
// cvode.max_substeps): b200.lu_fp64, b200.kernel, and b200.surrogate =
// <weights file>, which selects the surrogate-first hybrid react
// (b200chem_react_hybrid_boxes) with the acceptance rule stored in the file.
#pragma once

#include <string>
#include <vector>

#include "ReactorBase.H"
#include "b200chem.h"

// The mechanism of the build as a flat description (defined by the build).
b200chem_mech_desc b200chem_make_mech_desc();

namespace pele::physics::reactions {

// Array4 -> b200chem view: base pointer, strides, and the fab's index box.
template <class A4>
inline b200chem_array4 b200chem_view(A4 const& a) {
  b200chem_array4 r{};
  r.p = const_cast<double*>(static_cast<const double*>(a.p));
  r.jstride = a.jstride;
  r.kstride = a.kstride;
  r.nstride = a.nstride;
  for (int d = 0; d < 3; ++d) {
    r.lo[d] = a.begin[d];
    r.hi[d] = a.end[d] - 1;
  }
  return r;
}

template <class A4>
inline b200chem_iarray4 b200chem_iview(A4 const& a) {
  b200chem_iarray4 r{};
  r.p = a.p;
  r.jstride = a.jstride;
  r.kstride = a.kstride;
  r.nstride = a.nstride;
  for (int d = 0; d < 3; ++d) {
    r.lo[d] = a.begin[d];
    r.hi[d] = a.end[d] - 1;
  }
  return r;
}

class ReactorB200 : public ReactorBase::Register<ReactorB200> {
public:
  static std::string identifier() { return "ReactorB200"; }

  int init(int reactor_type, int /*ncells*/) override {
    amrex::ParmParse pp("ode"), pc("cvode"), pb("b200");
    b200chem_opts o{};
    o.rtol = 1e-10;  // the reference's defaults (LMeXControls.rst:301-310)
    o.atol = 1e-10;
    o.max_order = 2;
    o.max_steps = 10000;
    pp.query("rtol", o.rtol);
    pp.query("atol", o.atol);
    pc.query("max_order", o.max_order);
    pc.query("max_substeps", o.max_steps);
    pb.query("lu_fp64", o.lu_fp64);
    pb.query("kernel", o.kernel);
    pb.query("refine_stall_ppm", o.refine_stall_ppm);
    pb.query("refine_keep_ppm", o.refine_keep_ppm);
    o.reactor_type = reactor_type;  // 2: HP
    const b200chem_mech_desc d = b200chem_make_mech_desc();
    h_ = b200chem_create(&d, &o);
    if (!h_) amrex::Abort(b200chem_last_error());
    std::string weights;
    pb.query("surrogate", weights);
    if (!weights.empty()) {
      sur_ = b200chem_surrogate_load_file(h_, weights.c_str());
      if (!sur_) amrex::Abort(b200chem_last_error());
    }
    return 0;
  }

  // The library takes its thermodynamics from the mechanism description
  // (ideal gas, NASA-7), so the EOS parameters are kept but not read.
  void set_eos_parm(const pele::physics::eos::EosParm<pele::physics::PhysicsType::eos_type>* p) override {
    eos_parm_ = p;
  }

  void set_typ_vals_ode(const std::vector<amrex::Real>& v) override {
    if (b200chem_set_typvals(h_, v.data(), static_cast<int32_t>(v.size())) != 0) amrex::Abort(b200chem_last_error());
  }

  int react(const amrex::Box& box, amrex::Array4<amrex::Real> const& rY, amrex::Array4<amrex::Real> const& rYsrc,
            amrex::Array4<amrex::Real> const& T, amrex::Array4<amrex::Real> const& rE,
            amrex::Array4<amrex::Real> const& rEsrc, amrex::Array4<amrex::Real> const& fc,
            amrex::Array4<int> const& mask, amrex::Real& dt_react, amrex::Real& time,
            amrex::gpuStream_t stream) override {
    const b200chem_box_view v = box_view(box, rY, rYsrc, T, rE, rEsrc, fc, mask);
    void* st = reinterpret_cast<void*>(stream);
    // the reference aborts the run when its integrator fails
    const int rc = sur_ ? b200chem_react_hybrid_boxes(h_, sur_, nullptr, &v, 1, &dt_react, &time, st, nullptr,
                                                      nullptr, nullptr)
                        : b200chem_react(h_, &v, 1, &dt_react, &time, st, nullptr, nullptr);
    if (rc != 0) amrex::Abort(b200chem_last_error());
    return 0;
  }

  void close() override {
    b200chem_surrogate_destroy(sur_);
    sur_ = nullptr;
    b200chem_destroy(h_);
    h_ = nullptr;
  }

  bool hybrid() const { return sur_ != nullptr; }

  // The b200chem view of one react call's box and fabs.
  static b200chem_box_view box_view(const amrex::Box& box, amrex::Array4<amrex::Real> const& rY,
                                    amrex::Array4<amrex::Real> const& rYsrc, amrex::Array4<amrex::Real> const& T,
                                    amrex::Array4<amrex::Real> const& rE, amrex::Array4<amrex::Real> const& rEsrc,
                                    amrex::Array4<amrex::Real> const& fc, amrex::Array4<int> const& mask) {
    b200chem_box_view v{};
    for (int d = 0; d < 3; ++d) {
      v.lo[d] = box.smallEnd(d);
      v.hi[d] = box.bigEnd(d);
    }
    v.rhoY = b200chem_view(rY);
    v.extF_rhoY = b200chem_view(rYsrc);
    v.T = b200chem_view(T);
    v.rhoH = b200chem_view(rE);
    v.extF_rhoH = b200chem_view(rEsrc);
    v.fctCount = b200chem_view(fc);
    v.mask = b200chem_iview(mask);
    return v;
  }

private:
  b200chem_handle h_ = nullptr;
  b200chem_surrogate_handle sur_ = nullptr;
  const pele::physics::eos::EosParm<pele::physics::PhysicsType::eos_type>* eos_parm_ = nullptr;
};

}  // namespace pele::physics::reactions
