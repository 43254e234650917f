// Oracle heap fast-marching solve of one region (the reference algorithm the
// device fixed-point solver is checked against).  TEST INFRASTRUCTURE ONLY.
#include "oracle.hpp"
#include <stdexcept>
#include <algorithm>

namespace orc {

namespace {

// State that propagate2d.f90 keeps in module mod_prop2d (:1-30).
struct Fmm {
  Model* m;
  Region* r;
  const Grid* g;
  std::vector<double> vel;                 // copy of region velocity
  std::vector<int> tree;                   // node_from_tree_ind (1-based)
  std::vector<int> counted;                // node_is_counted
  std::vector<uint8_t> suspect;            // suspect_time_gradient
  int ntree = 0, newalive = 0;
  int n_connode = 0, n_concell = 0;
  int connode[128];
  int cc_ix[4], cc_iz[4], cc_nnode[4], cc_nbase[4];
  bool cc_reg[4];
  long n_det_negative = 0;

  int rid(int ix, int iz) const { return r->rid[g->g(ix, iz)]; }

  // ---------------------------------------------------------------- heap
  // propagate2d.f90:1199-1332 — binary min-heap keyed on arrival time with
  // back-pointers in node_status.
  void add(int nn) {
    ++ntree;
    r->status[nn] = ntree;
    tree[ntree] = nn;
    int child = ntree, parent = ntree / 2;
    while (parent > 0) {
      if (r->T[nn] < r->T[tree[parent]]) {
        r->status[nn] = parent;
        r->status[tree[parent]] = child;
        std::swap(tree[child], tree[parent]);
        child = parent;
        parent = child / 2;
      } else {
        parent = 0;
      }
    }
  }
  void remove_root() {
    if (ntree == 1) { ntree = 0; return; }
    r->status[tree[ntree]] = 1;
    tree[1] = tree[ntree];
    --ntree;
    int parent = 1, child = 2;
    while (child < ntree) {
      if (r->T[tree[child]] > r->T[tree[child + 1]]) ++child;
      if (r->T[tree[child]] < r->T[tree[parent]]) {
        r->status[tree[parent]] = child;
        r->status[tree[child]] = parent;
        std::swap(tree[child], tree[parent]);
        parent = child;
        child = 2 * parent;
      } else {
        child = ntree + 1;
      }
    }
    if (child == ntree) {
      if (r->T[tree[child]] < r->T[tree[parent]]) {
        r->status[tree[parent]] = child;
        r->status[tree[child]] = parent;
        std::swap(tree[child], tree[parent]);
      }
    }
  }
  void update_tree(int nn) {
    int child = r->status[nn], parent = child / 2;
    while (parent > 0) {
      if (r->T[nn] < r->T[tree[parent]]) {
        r->status[nn] = parent;
        r->status[tree[parent]] = child;
        std::swap(tree[child], tree[parent]);
        child = parent;
        parent = child / 2;
      } else {
        parent = 0;
      }
    }
  }

  void push_con(int mm) {
    if (n_connode >= 128) throw std::runtime_error("connode overflow");
    connode[n_connode++] = mm;
  }

  // Cells around a node: the (up to) four grid cells of a grid node, or the
  // cut cells listed for an interface node (propagate2d.f90:160-195).
  void concells_of(int cn) {
    const int i1 = r->i1[cn], i2 = r->i2[cn], i3 = r->i3[cn];
    n_concell = 0;
    if (i1 != 0) {
      for (int i = 0; i <= 1; ++i)
        if (i1 - i > 0 && i1 - i < g->nx)
          for (int j = 0; j <= 1; ++j)
            if (i2 - j > 0 && i2 - j < g->nz) {
              cc_ix[n_concell] = i1 - i;
              cc_iz[n_concell] = i2 - j;
              ++n_concell;
            }
    } else {
      const Isec& is = m->isec[i2 == r->itop ? r->itop : r->ibot];
      for (int k = 1; k <= 4; ++k) {
        const int c = is.ccfi(k, i3);
        if (c > 0) {
          cc_ix[n_concell] = is.cc_ix[c];
          cc_iz[n_concell] = is.cc_iz[c];
          ++n_concell;
        }
      }
    }
  }

  // propagate2d.f90:130-339
  void find_connected_nodes(int cn) {
    const int i1 = r->i1[cn], i2 = r->i2[cn];
    if (i1 != 0 && g->fully_regular[g->g(i1, i2)]) {
      n_connode = 0;
      if (rid(i1 - 1, i2) > 0) push_con(rid(i1 - 1, i2));
      if (rid(i1 + 1, i2) > 0) push_con(rid(i1 + 1, i2));
      if (rid(i1, i2 - 1) > 0) push_con(rid(i1, i2 - 1));
      if (rid(i1, i2 + 1) > 0) push_con(rid(i1, i2 + 1));
      return;
    }
    concells_of(cn);
    counted[cn] = cn;
    n_connode = 0;
    auto add_once = [&](int mm) {
      if (counted[mm] != cn) { push_con(mm); counted[mm] = cn; }
    };
    for (int n = 0; n < n_concell; ++n) {
      cc_reg[n] = (i1 != 0);
      const int gi = g->g(cc_ix[n], cc_iz[n]);
      if (g->cc_assoc[gi]) {
        int c = g->cc_idx[(size_t)gi * 6 + r->itop];
        if (c != 0) {
          cc_reg[n] = false;
          const Isec& is = m->isec[r->itop];
          for (int jj = 1; jj <= is.n_inodes[c]; ++jj) add_once(r->itop_rid[is.inode(jj, c)]);
        }
        c = g->cc_idx[(size_t)gi * 6 + r->ibot];
        if (c != 0) {
          cc_reg[n] = false;
          const Isec& is = m->isec[r->ibot];
          for (int jj = 1; jj <= is.n_inodes[c]; ++jj) add_once(r->ibot_rid[is.inode(jj, c)]);
        }
      }
      for (int i = 0; i <= 1; ++i) {
        const int ii = cc_ix[n] + i;
        for (int j = 0; j <= 1; ++j) {
          const int jj = cc_iz[n] + j;
          if (ii >= 1 && ii <= g->nx && jj >= 1 && jj <= g->nz) {
            if ((i1 != 0 && std::abs(i1 - ii) + std::abs(i2 - jj) == 1) || !cc_reg[n]) {
              const int mm = rid(ii, jj);
              if (mm > 0) add_once(mm);
            }
          }
        }
      }
    }
    if (i1 == 0) {
      // fallback search for grid nodes next to an interface node
      int ix = (int)std::lround((r->x[cn] - g->x0) / g->dx) + 1;
      ix = std::max(1, std::min(g->nx, ix));
      int izs = (int)std::lround((r->z[cn] - g->z0) / g->dz) + 1;
      izs = std::max(1, std::min(g->nz, izs));
      if (i2 == r->ibot) {
        for (int ixx = std::max(1, ix - 1); ixx <= std::min(g->nx, ix + 1); ++ixx)
          for (int izz = izs; izz >= 1; --izz) {
            const int mm = rid(ixx, izz);
            if (mm > 0) { add_once(mm); break; }
          }
      } else {
        for (int ixx = std::max(1, ix - 1); ixx <= std::min(g->nx, ix + 1); ++ixx)
          for (int izz = izs; izz <= g->nz; ++izz) {
            const int mm = rid(ixx, izz);
            if (mm > 0) { add_once(mm); break; }
          }
      }
    }
  }

  // propagate2d.f90:342-479 — accepted nodes per connected cell.
  void find_connected_cells(int cn) {
    const int i1 = r->i1[cn], i2 = r->i2[cn];
    concells_of(cn);
    n_connode = 0;
    for (int n = 0; n < n_concell; ++n) {
      cc_reg[n] = (i1 != 0);
      const int gi = g->g(cc_ix[n], cc_iz[n]);
      if (g->cc_assoc[gi]) {
        int c = g->cc_idx[(size_t)gi * 6 + r->itop];
        if (c != 0) {
          cc_reg[n] = false;
          const Isec& is = m->isec[r->itop];
          for (int jj = 1; jj <= is.n_inodes[c]; ++jj) {
            const int mm = r->itop_rid[is.inode(jj, c)];
            if (r->status[mm] == 0) push_con(mm);
          }
        }
        c = g->cc_idx[(size_t)gi * 6 + r->ibot];
        if (c != 0) {
          cc_reg[n] = false;
          const Isec& is = m->isec[r->ibot];
          for (int jj = 1; jj <= is.n_inodes[c]; ++jj) {
            const int mm = r->ibot_rid[is.inode(jj, c)];
            if (r->status[mm] == 0) push_con(mm);
          }
        }
      }
      for (int i = 0; i <= 1; ++i) {
        const int ii = cc_ix[n] + i;
        for (int j = 0; j <= 1; ++j) {
          const int jj = cc_iz[n] + j;
          if (ii < 1 || ii > g->nx || jj < 1 || jj > g->nz) continue;
          if ((i1 != 0 && std::abs(i1 - ii) + std::abs(i2 - jj) == 1) || !cc_reg[n]) {
            const int mm = rid(ii, jj);
            if (mm > 0 && mm <= r->nnode && r->status[mm] == 0) push_con(mm);
          }
        }
      }
      cc_nnode[n] = n_connode;
    }
    cc_nbase[0] = 1;
    for (int n = 0; n < n_concell; ++n) {
      cc_nnode[n] = cc_nnode[n] - cc_nbase[n] + 1;
      if (n < n_concell - 1) cc_nbase[n + 1] = cc_nbase[n] + cc_nnode[n];
    }
  }

  // propagate2d.f90:605-790
  void regular_update(int un, const int* an, int na) {
    if (na > 2) throw std::runtime_error("too many nodes for regular update2d");
    const int iu = r->i1[un], ju = r->i2[un];
    double a = 0, b = 0, c = 0, t2x = 0, t2z = 0, tx = 0, tz = 0, tmax = 0;
    bool xi = false, zi = false;
    int ioff = 0, joff = 0;
    for (int n = 0; n < na; ++n) {
      const int nd = an[n];
      tmax = std::max(tmax, r->T[nd]);
      const int ia = r->i1[nd], ja = r->i2[nd];
      if (ia == 0) continue;
      if (ia != iu) {
        xi = true;
        ioff = ia;
        const int di = ia - iu, ias = iu + 2 * di;
        const double velx = 0.5 * (vel[un] + vel[nd]);
        bool second = false;
        if (ias >= 1 && ias <= g->nx && rid(ias, ja) > 0) {
          const int sn = rid(ias, ja);
          if (sn > 0 && sn <= r->nnode && r->status[sn] == 0 && r->T[nd] >= r->T[sn]) {
            if (vel[nd] * vel[sn] > kTiny &&
                r->gx[nd] * r->gx[sn] + r->gz[nd] * r->gz[sn] >= 0.71 / (vel[nd] * vel[sn])) {
              tx = r->T[nd];
              t2x = r->T[sn];
              const double d2 = (velx / g->dx) * (velx / g->dx);
              a += 2.25 * d2;
              b += (-6.0 * tx + 1.5 * t2x) * d2;
              c += (4.0 * tx * tx - 2.0 * tx * t2x + 0.25 * t2x * t2x) * d2;
              second = true;
            }
          }
        }
        if (second) continue;
        tx = r->T[nd];
        const double d2 = (velx / g->dx) * (velx / g->dx);
        a += d2;
        b += (-2.0 * tx) * d2;
        c += (tx * tx) * d2;
      } else if (ja != ju) {
        zi = true;
        joff = ja;
        const int dj = ja - ju, jas = ju + 2 * dj;
        const double velz = 0.5 * (vel[un] + vel[nd]);
        bool second = false;
        if (jas >= 1 && jas <= g->nz && rid(ia, jas) > 0) {
          const int sn = rid(ia, jas);
          if (sn > 0 && sn <= r->nnode && r->status[sn] == 0 && r->T[nd] >= r->T[sn]) {
            if (vel[nd] * vel[sn] > kTiny &&
                r->gx[nd] * r->gx[sn] + r->gz[nd] * r->gz[sn] >= 0.71 / (vel[nd] * vel[sn])) {
              tz = r->T[nd];
              t2z = r->T[sn];
              const double d2 = (velz / g->dz) * (velz / g->dz);
              a += 2.25 * d2;
              b += (-6.0 * tz + 1.5 * t2z) * d2;
              c += (4.0 * tz * tz - 2.0 * tz * t2z + 0.25 * t2z * t2z) * d2;
              second = true;
            }
          }
        }
        if (second) continue;
        tz = r->T[nd];
        const double d2 = (velz / g->dz) * (velz / g->dz);
        a += d2;
        b += (-2.0 * tz) * d2;
        c += (tz * tz) * d2;
      }
    }
    c = c - 1.0;
    if (std::fabs(a) < kTiny) return;
    double det = b * b - 4.0 * a * c;
    if (det < 0.0) {
      if (0.5 * std::sqrt(std::fabs(det)) / std::fabs(a) < 1.0e20) {
        det = 0.0;
        ++n_det_negative;
      } else {
        throw std::runtime_error("negative determinant too large");
      }
    }
    double t1 = 0.5 * (-b + std::sqrt(det)) / a;
    t1 = std::max(t1, tmax);
    if (t1 < r->T[un]) {
      r->T[un] = t1;
      r->gx[un] = 0.0;
      r->gz[un] = 0.0;
      if (xi) {
        if (t2x == 0.0) r->gx[un] = (t1 - tx) / (g->x[iu] - g->x[ioff]);
        else r->gx[un] = 0.5 * (3.0 * t1 - 4.0 * tx + t2x) / (g->x[iu] - g->x[ioff]);
      }
      if (zi) {
        if (t2z == 0.0) r->gz[un] = (t1 - tz) / (g->z[ju] - g->z[joff]);
        else r->gz[un] = 0.5 * (3.0 * t1 - 4.0 * tz + t2z) / (g->z[ju] - g->z[joff]);
      }
      suspect[un] = !(xi && zi);
    }
  }

  // propagate2d.f90:793-829
  void time_from_1(int un, int n1) {
    const double dxu = r->x[un] - r->x[n1], dzu = r->z[un] - r->z[n1];
    const double dist = std::sqrt(dxu * dxu + dzu * dzu);
    if (dist < 0.01 * g->tolerance) {
      r->T[un] = r->T[n1];
      r->gx[un] = r->gx[n1];
      r->gz[un] = r->gz[n1];
      return;
    }
    const double tt = dist / (0.5 * (vel[un] + vel[n1]));
    const double at = r->T[n1] + tt;
    if (at < r->T[un]) {
      r->T[un] = at;
      r->gx[un] = dxu / (dist * vel[un]);
      r->gz[un] = dzu / (dist * vel[un]);
    }
  }

  // propagate2d.f90:832-946
  void time_from_2(int un, int a1, int a2) {
    int n1 = a1, n2 = a2;
    if (r->T[n1] < r->T[n2]) std::swap(n1, n2);
    const double xu = r->x[un], zu = r->z[un];
    const double r1x = r->x[n1] - xu, r1z = r->z[n1] - zu;
    const double r2x = r->x[n2] - xu, r2z = r->z[n2] - zu;
    if (std::sqrt(r1x * r1x + r1z * r1z) < 0.01 * g->tolerance) {
      r->T[un] = r->T[n1]; r->gx[un] = r->gx[n1]; r->gz[un] = r->gz[n1];
      return;
    }
    if (std::sqrt(r2x * r2x + r2z * r2z) < 0.01 * g->tolerance) {
      r->T[un] = r->T[n2]; r->gx[un] = r->gx[n2]; r->gz[un] = r->gz[n2];
      return;
    }
    const double ex = r->x[n2] - r->x[n1], ez = r->z[n2] - r->z[n1];
    if (std::sqrt(ex * ex + ez * ez) < 0.01 * g->tolerance) { time_from_1(un, n1); return; }
    const double v12 = 0.5 * (vel[n1] + vel[n2]);
    const double dx_ = (r->x[n1] - r->x[n2]) / v12, dz_ = (r->z[n1] - r->z[n2]) / v12;
    const double dd = dx_ * dx_ + dz_ * dz_;
    const double px = (r->T[n1] - r->T[n2]) / dd * dx_;
    const double pz = (r->T[n1] - r->T[n2]) / dd * dz_;
    const double qx = -dz_, qz = dx_;
    const double ae = qx * qx + qz * qz;
    const double be = 2.0 * (px * qx + pz * qz);
    const double ce = px * px + pz * pz - 1.0;
    const double det = be * be - 4.0 * ae * ce;
    if (det < 0.0) return;
    const double u1 = 0.5 * (-be + std::sqrt(det)) / ae;
    const double u2 = 0.5 * (-be - std::sqrt(det)) / ae;
    const double w1x = px + u1 * qx, w1z = pz + u1 * qz;
    const double w2x = px + u2 * qx, w2z = pz + u2 * qz;
    double n1x = -r1z, n1z = r1x;
    double l = std::sqrt(n1x * n1x + n1z * n1z);
    n1x /= l; n1z /= l;
    if (n1x * r2x + n1z * r2z < 0.0) { n1x = -n1x; n1z = -n1z; }
    double n2x = -r2z, n2z = r2x;
    l = std::sqrt(n2x * n2x + n2z * n2z);
    n2x /= l; n2z /= l;
    if (n2x * r1x + n2z * r1z < 0.0) { n2x = -n2x; n2z = -n2z; }
    auto try_w = [&](double wx, double wz) {
      if (wx * n1x + wz * n1z <= 0.0 && wx * n2x + wz * n2z <= 0.0) {
        const double at = r->T[n1] - (wx * r1x + wz * r1z) / (0.5 * (vel[un] + vel[n1]));
        if (at >= r->T[n1]) {
          if (at < r->T[un]) {
            r->T[un] = at;
            const double wl = std::sqrt(wx * wx + wz * wz);
            r->gx[un] = wx / (wl * vel[n1]);
            r->gz[un] = wz / (wl * vel[n1]);
          }
        }
      }
    };
    try_w(w1x, w1z);
    try_w(w2x, w2z);
  }

  // propagate2d.f90:482-602
  void update_time(int un) {
    const int i1 = r->i1[un], i2 = r->i2[un];
    if (i1 != 0 && g->fully_regular[g->g(i1, i2)]) {
      for (int j = -1; j <= 1; j += 2) {
        for (int i = -1; i <= 1; i += 2) {
          int an[2], na = 0;
          int id = rid(i1 + i, i2);
          if (id > 0 && id <= r->nnode && r->status[id] == 0) an[na++] = id;
          id = rid(i1, i2 + j);
          if (id > 0 && id <= r->nnode && r->status[id] == 0) an[na++] = id;
          if (na > 0) {
            for (int n = 0; n < na; ++n)
              if (an[n] == newalive) { an[n] = an[0]; an[0] = newalive; }
            if (an[0] == newalive) regular_update(un, an, na);
          }
        }
      }
      return;
    }
    find_connected_cells(un);
    int an[30];
    for (int n = 0; n < n_concell; ++n) {
      if (cc_nnode[n] <= 0) continue;
      const int na = cc_nnode[n];
      if (na > 30) throw std::runtime_error("update_time2d: nanode > 30");
      for (int k = 0; k < na; ++k) an[k] = connode[cc_nbase[n] - 1 + k];
      for (int k = 0; k < na; ++k)
        if (an[k] == newalive) std::swap(an[0], an[k]);
      if (an[0] != newalive) continue;
      if (cc_reg[n]) {
        regular_update(un, an, na);
      } else {
        time_from_1(un, an[0]);
        for (int k = 1; k < na; ++k) time_from_2(un, an[0], an[k]);
      }
    }
  }

  // propagate2d.f90:33-127
  void run() {
    const int nn = r->nnode;
    vel.assign(r->vel.begin(), r->vel.end());
    suspect.assign(nn + 1, 0);
    tree.assign(nn + 2, 0);
    counted.assign(nn + 1, 0);
    ntree = 0;
    for (int n = 1; n <= nn; ++n)
      if (r->status[n] > 0) add(n);
    bool first = true;
    while (ntree > 0) {
      newalive = tree[1];
      r->status[newalive] = 0;
      remove_root();
      if (ntree == 0 && !first) break;
      first = false;
      find_connected_nodes(newalive);
      int trial[128];
      const int nt = n_connode;
      for (int k = 0; k < nt; ++k) trial[k] = connode[k];
      for (int k = 0; k < nt; ++k) {
        const int tn = trial[k];
        if (r->status[tn] > 0) {
          const double old = r->T[tn];
          update_time(tn);
          if (r->T[tn] < old) update_tree(tn);
        }
        if (r->status[tn] == -1) {
          r->T[tn] = kHugeTime;
          const double old = r->T[tn];
          update_time(tn);
          if (r->T[tn] < old) add(tn);
        }
      }
    }
    for (int n = 1; n <= nn; ++n)
      if (suspect[n]) fit_gradient_at_node2d(*m, *r, n, r->gx[n], r->gz[n]);
  }
};

}  // namespace

void propagate2d(Model& m, Region& r) {
  Fmm f;
  f.m = &m;
  f.r = &r;
  f.g = &m.grid;
  f.run();
}

// propagate2d.f90:949-1196 — central differences on regular neighbourhoods,
// otherwise a distance-weighted 2x2 least-squares fit over nearby nodes.
void fit_gradient_at_node2d(const Model& m, const Region& r, int cn, double& dtdx,
                            double& dtdz) {
  const Grid& g = m.grid;
  const int i1 = r.i1[cn], i2 = r.i2[cn], i3 = r.i3[cn];
  int ncl = 0, clx[4], clz[4];
  if (i1 != 0) {
    for (int i = 0; i <= 1; ++i)
      if (i1 - i > 0 && i1 - i < g.nx)
        for (int j = 0; j <= 1; ++j)
          if (i2 - j > 0 && i2 - j < g.nz) { clx[ncl] = i1 - i; clz[ncl] = i2 - j; ++ncl; }
  } else {
    const Isec& is = m.isec[i2 == r.itop ? r.itop : r.ibot];
    for (int k = 1; k <= 4; ++k) {
      const int c = is.ccfi(k, i3);
      if (c > 0) { clx[ncl] = is.cc_ix[c]; clz[ncl] = is.cc_iz[c]; ++ncl; }
    }
  }
  bool irr[4];
  int nirr = 0;
  for (int n = 0; n < ncl; ++n) {
    irr[n] = g.cc_assoc[g.g(clx[n], clz[n])] != 0;
    nirr += irr[n] ? 1 : 0;
  }
  auto rid = [&](int ix, int iz) { return r.rid[g.g(ix, iz)]; };
  if (nirr == 0) {
    if (i1 != 0) {
      int mm = rid(std::max(1, i1 - 1), i2), nn = rid(std::min(g.nx, i1 + 1), i2);
      const bool okm = mm > 0 && mm <= r.nnode, okn = nn > 0 && nn <= r.nnode;
      if (okm && okn) dtdx = (r.T[nn] - r.T[mm]) / (r.x[nn] - r.x[mm]);
      else if (okm) dtdx = (r.T[cn] - r.T[mm]) / (r.x[cn] - r.x[mm]);
      else if (okn) dtdx = (r.T[nn] - r.T[cn]) / (r.x[nn] - r.x[cn]);
      else dtdx = 0.0;
      mm = rid(i1, std::max(1, i2 - 1));
      nn = rid(i1, std::min(g.nz, i2 + 1));
      const bool okm2 = mm > 0 && mm <= r.nnode, okn2 = nn > 0 && nn <= r.nnode;
      if (okm2 && okn2) dtdz = (r.T[nn] - r.T[mm]) / (r.z[nn] - r.z[mm]);
      else if (okm2) dtdz = (r.T[cn] - r.T[mm]) / (r.z[cn] - r.z[mm]);
      else if (okn2) dtdz = (r.T[nn] - r.T[cn]) / (r.z[nn] - r.z[cn]);
      else dtdz = 0.0;
      return;
    }
    if (ncl == 0) { dtdx = 0.0; dtdz = 0.0; return; }
  }
  const int maxfit = 30;
  int ncn = 0, store[30];
  double rx[30], rz[30], at[30];
  auto take = [&](int mm) {
    if (mm == cn) return;
    for (int k = 0; k < ncn; ++k)
      if (store[k] == mm) return;
    if (ncn < maxfit) {
      store[ncn] = mm; rx[ncn] = r.x[mm]; rz[ncn] = r.z[mm]; at[ncn] = r.T[mm];
      ++ncn;
    }
  };
  for (int n = 0; n < ncl; ++n) {
    if (irr[n]) {
      const int gi = g.g(clx[n], clz[n]);
      int c = g.cc_idx[(size_t)gi * 6 + r.itop];
      if (c != 0) {
        const Isec& is = m.isec[r.itop];
        for (int jj = 1; jj <= is.n_inodes[c]; ++jj) take(r.itop_rid[is.inode(jj, c)]);
      }
      c = g.cc_idx[(size_t)gi * 6 + r.ibot];
      if (c != 0) {
        const Isec& is = m.isec[r.ibot];
        for (int jj = 1; jj <= is.n_inodes[c]; ++jj) take(r.ibot_rid[is.inode(jj, c)]);
      }
    }
    for (int i = 0; i <= 1; ++i) {
      const int ii = clx[n] + i;
      if (ii < 1 || ii > g.nx) continue;
      for (int j = 0; j <= 1; ++j) {
        const int jj = clz[n] + j;
        if (jj < 1 || jj > g.nz) continue;
        const int mm = rid(ii, jj);
        if (mm <= 0 || mm > r.nnode) continue;
        take(mm);
      }
    }
  }
  double a11 = 0, a12 = 0, a22 = 0, b1 = 0, b2 = 0;
  for (int i = 0; i < ncn; ++i) {
    const double ddx = rx[i] - r.x[cn], ddz = rz[i] - r.z[cn];
    const double dw = 1.0 / (std::sqrt(ddx * ddx + ddz * ddz) + g.tolerance);
    a11 += ddx * ddx * dw * dw;
    a12 += ddx * ddz * dw * dw;
    a22 += ddz * ddz * dw * dw;
    b1 += (at[i] - r.T[cn]) * ddx * dw * dw;
    b2 += (at[i] - r.T[cn]) * ddz * dw * dw;
  }
  const double det = a11 * a22 - a12 * a12;
  if (std::fabs(det) < 1.0e-30) { dtdx = 0.0; dtdz = 0.0; return; }
  dtdx = (a22 * b1 - a12 * b2) / det;
  dtdz = (a11 * b2 - a12 * b1) / det;
}

}  // namespace orc
