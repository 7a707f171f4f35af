// lulesh.hpp -- C++ host interface mirroring the reference's LULESH API,
// implemented over the C ABI of include/lulesh_b200.h.
//
// Reference names kept (LULESH/cuda/src/lulesh.h, lulesh.cu):
//   Domain, NewDomain, LagrangeLeapFrog, VerifyAndWriteFinalOutput numbers,
//   CommRecv / CommSend / CommSBN / CommSyncPosVel / CommMonoQ, the message
//   tags MSG_COMM_SBN / MSG_SYNC_POS_VEL / MSG_MONOQ and the error codes
//   VolumeError / QStopError / LFileError.
// A Domain here is one rank of a set that lives on one GPU: rank r of a
// tp^3 decomposition is subdomain r of the set, and the Comm* calls move
// halos between subdomains in device memory (numRanks() == 1 makes them
// no-ops, as lulesh-comms.cu:65-66 does).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "lulesh_b200.h"

namespace lulesh_b200 {

enum { VolumeError = -1, QStopError = -2, LFileError = -3 };  // lulesh.h:22-26

constexpr int MSG_COMM_SBN = LULESH_MSG_COMM_SBN;         // lulesh.h:315
constexpr int MSG_SYNC_POS_VEL = LULESH_MSG_SYNC_POS_VEL; // lulesh.h:316
constexpr int MSG_MONOQ = LULESH_MSG_MONOQ;               // lulesh.h:317

typedef int Index_t;
typedef int Int_t;
typedef double Real_t;

// the reference passes Domain member-function pointers (Domain_member,
// lulesh.h:300); here a field is named by its lulesh_field_id
typedef int Domain_member;

class Error : public std::runtime_error {
  public:
    Error(int st, const std::string &what)
        : std::runtime_error(what + ": " + lulesh_status_string(st) + " " + lulesh_last_error()),
          status(st)
    {
    }
    int status;
};

inline void check(int st, const char *what)
{
    if (st != LULESH_OK) throw Error(st, what);
}

// Owns the GPU-resident set (all ranks of one problem).
class DomainSet {
  public:
    DomainSet(int nx, int tp, int nr, int balance, int cost, int its, int flags, int device = -1)
    {
        lulesh_job j{nx, nr, balance, cost, its};
        check(lulesh_create(&j, tp, flags, device, &set_), "NewDomain");
        tp_ = tp;
    }
    // NewDomain's unstructured branch: one domain read from an lmesh file
    DomainSet(const char *mesh, int nr, int balance, int cost, int its, int flags,
              int device = -1)
    {
        lulesh_job j{1, nr, balance, cost, its};
        check(lulesh_create_from_mesh(mesh, &j, flags, device, &set_), "NewDomain");
    }
    ~DomainSet() { release(); }
    // free every device resource now (the destructor then does nothing)
    void release()
    {
        if (set_) lulesh_destroy(set_);
        set_ = nullptr;
    }
    DomainSet(const DomainSet &) = delete;
    DomainSet &operator=(const DomainSet &) = delete;
    lulesh_set *get() const { return set_; }
    int tp() const { return tp_; }

  private:
    lulesh_set *set_ = nullptr;
    int tp_ = 1;
};

// One rank's view (lulesh.h:40-298 member names through view()).
class Domain {
  public:
    Domain(DomainSet &set, int rank) : set_(&set), rank_(rank)
    {
        check(lulesh_domain_view_get(set.get(), rank, &view_), "Domain view");
    }
    const lulesh_domain_view &view() const { return view_; }
    lulesh_set *set() const { return set_->get(); }
    int rank() const { return rank_; }
    Index_t numRanks() const { return set_->tp() * set_->tp() * set_->tp(); }
    Index_t &colLoc() { return view_.colLoc; }
    Index_t &rowLoc() { return view_.rowLoc; }
    Index_t &planeLoc() { return view_.planeLoc; }
    Index_t &tp() { return view_.tp; }
    Index_t numElem() const { return view_.numElem; }
    Index_t numNode() const { return view_.numNode; }
    Index_t sizeX() const { return view_.sizeX; }

    std::vector<Real_t> field(const char *name) const
    {
        size_t nb = 0;
        check(lulesh_field_bytes(set(), rank_, name, &nb), "field size");
        std::vector<Real_t> v(nb / sizeof(Real_t));
        check(lulesh_get_field(set(), rank_, name, v.data(), nb), "get field");
        return v;
    }
    lulesh_job_state state() const
    {
        lulesh_job_state s;
        check(lulesh_job_state_get(set(), 0, &s), "job state");
        return s;
    }
    Real_t time() const { return state().time; }
    Real_t deltatime() const { return state().deltatime; }
    Int_t cycle() const { return state().cycle; }

  private:
    DomainSet *set_;
    int rank_;
    lulesh_domain_view view_{};
};

// TimeIncrement + LagrangeLeapFrog of every rank (lulesh.cu:4438-4452);
// asynchronous, like the reference's kernel launches.
inline void LagrangeLeapFrog(Domain *domain) { check(lulesh_lagrange_leapfrog(domain->set()), "LagrangeLeapFrog"); }

// comm backend, lulesh.h:321-340 (the *Gpu variants run on the set's stream)
inline void CommRecv(Domain &d, Int_t msgType, Index_t xferFields, Index_t dx, Index_t dy,
                     Index_t dz, bool doRecv, bool planeOnly)
{
    check(lulesh_comm_recv(d.set(), d.rank(), msgType, xferFields, dx, dy, dz, doRecv,
                           planeOnly),
          "CommRecv");
}
inline void CommSend(Domain &d, Int_t msgType, Index_t xferFields, Domain_member *fieldData,
                     Index_t dx, Index_t dy, Index_t dz, bool doSend, bool planeOnly)
{
    check(lulesh_comm_send(d.set(), d.rank(), msgType, xferFields, fieldData, dx, dy, dz, doSend,
                           planeOnly),
          "CommSend");
}
inline void CommSBN(Domain &d, Int_t xferFields, Domain_member *fieldData)
{
    check(lulesh_comm_sbn(d.set(), d.rank(), xferFields, fieldData), "CommSBN");
}
inline void CommSyncPosVel(Domain &d) { check(lulesh_comm_sync_posvel(d.set(), d.rank()), "CommSyncPosVel"); }
inline void CommMonoQ(Domain &d) { check(lulesh_comm_monoq(d.set(), d.rank()), "CommMonoQ"); }

}  // namespace lulesh_b200
