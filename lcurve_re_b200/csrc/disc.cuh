// disc.cuh — eclipses by a flared, cylindrically symmetric accretion disc.
//
// Restates Roche::disc_eclipse with its helpers circle_eclipse and cut_phase
// (disc_eclipse.cpp:38-366), in the reference's operation order, for the host
// engine and the kernels. The line of sight to a point sweeps a cone as the
// binary turns; where that cone meets the planes of the disc's rims, its
// intersection circle is compared with the rim circles, which gives the half
// width of the eclipse and, for points seen through the central hole, the
// half width of the window in which the point reappears.
#pragma once

#include "roche.cuh"

namespace lcg {

// Disc geometry for the eclipse test: sin and cos of the inclination as
// disc_eclipse computes them (sin(PI/180 * iangle)), inner and outer radius,
// flaring exponent and height at unit radius.
struct DiscGeom {
    double sini, cosi, rdisc1, rdisc2, beta, height;
};

enum { kCircAbove, kCircInside, kCircOutside, kCircSeparate, kCircCrossing };

// cut_phase (disc_eclipse.cpp:349-366); st = 3 (Roche_Error) when the two
// circles do not cross.
LCG_HD double cut_phase(double rxy, double rcone, double radius, int &st) {
    if (rxy + rcone <= radius || rxy >= radius + rcone || rcone >= radius + rxy) {
        st = 3;
        return 0.;
    }
    return acos((sq(rxy) + sq(rcone) - sq(radius)) / (2. * rcone * rxy)) / kTwoPi;
}

// circle_eclipse (disc_eclipse.cpp:316-340)
LCG_HD int circle_eclipse(double rxy, double z, double zcirc, double radius, double tani,
                          double &phase, int &st) {
    if (z >= zcirc) return kCircAbove;
    const double RCONE = tani * (zcirc - z);
    if (RCONE >= rxy + radius) return kCircOutside;
    if (rxy >= RCONE + radius) return kCircSeparate;
    if (rxy + RCONE <= radius) return kCircInside;
    phase = cut_phase(rxy, RCONE, radius, st);
    return kCircCrossing;
}

// Roche::disc_eclipse (disc_eclipse.cpp:38-301): appends 0, 1 or 2 phase
// ranges (in, out) during which the disc hides point r to rin/rout[nr...],
// up to cap entries. st = 3 on a Roche_Error (beta < 1 or a failed cut).
LCG_HD void disc_eclipse(const DiscGeom &g, V3 r, int &nr, double *rin, double *rout, int cap,
                         int &st) {
    auto push = [&](double a, double b) {
        if (nr < cap) {
            rin[nr] = a;
            rout[nr] = b;
        }
        nr++;
    };
    if (g.beta < 1) {
        st = 3;
        return;
    }
    const double HOUT = g.height * pow(g.rdisc2, g.beta);
    if (r.z >= HOUT) return;
    if (g.cosi == 0.) {
        if (fabs(r.z) < HOUT) {
            const double rxy = sqrt(sq(r.x) + sq(r.y));
            if (rxy <= g.rdisc2) {
                push(0., 1.);
            } else {
                const double subtend = asin(g.rdisc2 / rxy) / kTwoPi;
                const double pcen = atan2(r.y, -r.x) / kTwoPi;
                double ingress = pcen - subtend;
                ingress = ingress - floor(ingress);
                push(ingress, ingress + 2. * subtend);
            }
        }
        return;
    }
    const double RXY = sqrt(sq(r.x) + sq(r.y));
    if (g.rdisc1 < RXY && RXY < g.rdisc2 && fabs(r.z) < g.height * pow(RXY, g.beta)) {
        push(0., 1.1);
        return;
    }
    const double TANI = g.sini / g.cosi;
    int result;
    double phase = 0., ingress;
    if (RXY < g.rdisc2 && r.z >= g.height * pow((g.rdisc1 < RXY) ? RXY : g.rdisc1, g.beta)) {
        result = circle_eclipse(RXY, r.z, HOUT, g.rdisc2, TANI, phase, st);
        if (st) return;
        if (result == kCircOutside) {
            push(0., 1.1);
        } else if (result == kCircCrossing) {
            const double phi0 = atan2(r.y, -r.x) / kTwoPi;
            ingress = phi0 + phase;
            ingress -= floor(ingress);
            push(ingress, ingress + 1 - 2. * phase);
        }
        return;
    }
    const double lo = TANI * (-HOUT - r.z);
    const double RCONE_LO = (0. < lo) ? lo : 0.;
    if (RCONE_LO >= RXY + g.rdisc2) return;
    const double RCONE_HI = TANI * (HOUT - r.z);
    if (RXY >= RCONE_HI + g.rdisc2) return;
    double eclipse_phase = 0;
    if (RXY + RCONE_LO <= g.rdisc2) {
        eclipse_phase = 0.5;
    } else if (RXY <= g.rdisc2) {
        eclipse_phase = cut_phase(RXY, RCONE_LO, g.rdisc2, st);
    } else if (sq(RCONE_HI) + sq(g.rdisc2) >= sq(RXY) &&
               sq(RCONE_LO) + sq(g.rdisc2) <= sq(RXY)) {
        eclipse_phase = asin(g.rdisc2 / RXY) / kTwoPi;  // the curved outer rim
    } else if (sq(RCONE_HI) + sq(g.rdisc2) < sq(RXY)) {
        eclipse_phase = cut_phase(RXY, RCONE_HI, g.rdisc2, st);  // upper outer rim
    } else {
        eclipse_phase = cut_phase(RXY, RCONE_LO, g.rdisc2, st);  // lower outer rim
    }
    if (st) return;
    // Reappearance through the hole: the cone passes the rims below and
    // above the point in turn; the first fixes the window, each later one
    // can only narrow it or close it.
    const double HIN = g.height * pow(g.rdisc1, g.beta);
    double appear_phase = -1;
    double zc[4], rc[4];
    int nc = 0;
    if (r.z < -HOUT) {
        zc[0] = -HOUT; rc[0] = g.rdisc2; zc[1] = -HIN; rc[1] = g.rdisc1;
        zc[2] = HIN; rc[2] = g.rdisc1; zc[3] = HOUT; rc[3] = g.rdisc2;
        nc = 4;
    } else if (RXY < g.rdisc1) {
        if (r.z < -HIN) {
            zc[0] = -HIN; rc[0] = g.rdisc1; zc[1] = HIN; rc[1] = g.rdisc1;
            zc[2] = HOUT; rc[2] = g.rdisc2;
            nc = 3;
        } else if (r.z < HIN) {
            zc[0] = HIN; rc[0] = g.rdisc1; zc[1] = HOUT; rc[1] = g.rdisc2;
            nc = 2;
        }
    }
    for (int k = 0; k < nc; k++) {
        if (k > 0 && !(appear_phase > 0)) break;
        result = circle_eclipse(RXY, r.z, zc[k], rc[k], TANI, phase, st);
        if (st) return;
        if (k == 0) {
            if (result == kCircInside) appear_phase = 0.5;
            else if (result == kCircCrossing) appear_phase = phase;
        } else if (result == kCircCrossing) {
            appear_phase = (phase < appear_phase) ? phase : appear_phase;
        } else if (result != kCircInside) {
            appear_phase = -1.;
        }
    }
    const double phi0 = atan2(r.y, -r.x) / kTwoPi;
    if (appear_phase <= 0) {
        ingress = phi0 - eclipse_phase;
        ingress -= floor(ingress);
        push(ingress, ingress + 2. * eclipse_phase);
    } else if (appear_phase < eclipse_phase) {
        ingress = phi0 - eclipse_phase;
        ingress -= floor(ingress);
        push(ingress, ingress + (eclipse_phase - appear_phase));
        ingress = phi0 + appear_phase;
        ingress -= floor(ingress);
        push(ingress, ingress + (eclipse_phase - appear_phase));
    }
}

}  // namespace lcg
