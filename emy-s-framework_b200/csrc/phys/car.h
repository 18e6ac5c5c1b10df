// Car logic and vehicle model of one tick.
//
//   carPreTick ...... Car::_PreTickUpdate (Car.cpp:58-128) with btVehicleRL's
//                     updateVehicleFirst / updateVehicleSecond (btVehicleRL.cpp:208-230)
//   carPostTick ..... Car::_PostTickUpdate + Car::_FinishPhysicsTick (Car.cpp:130-193)
//   carRespawn ...... Car::Respawn (Car.cpp:44-56)
//
// Direction getters follow the reference: Car::GetForwardDir/GetRightDir/GetUpDir read
// CarState::rotMat (the basis saved by the last post-tick update), while btVehicleRL reads
// the chassis transform (forward axis 0, right axis 1, up axis 2).
//
// ALTERED SOURCE: this file is not the original Bullet code.  It restates the algorithms of
// the files named above (RocketSim's btVehicleRL derives from Bullet's btRaycastVehicle)
// for a CUDA device and a host build, with its own data layout, naming and control flow;
// the original's notice follows.
//
// Bullet Continuous Collision Detection and Physics Library
// Copyright (c) 2003-2006 Erwin Coumans  https://bulletphysics.org
//
// This software is provided 'as-is', without any express or implied warranty.
// In no event will the authors be held liable for any damages arising from the use of this software.
// Permission is granted to anyone to use this software for any purpose,
// including commercial applications, and to alter it and redistribute it freely,
// subject to the following restrictions:
//
// 1. The origin of this software must not be misrepresented; you must not claim that you wrote the original software. If you use this software in a product, an acknowledgment in the product documentation would be appreciated but is not required.
// 2. Altered source versions must be plainly marked as such, and must not be misrepresented as being the original software.
// 3. This notice may not be removed or altered from any source distribution.
#pragma once
#include "world.h"

namespace rsb {

// btRigidBody impulse / force helpers (btRigidBody.h:254-330), linear and angular factors 1
RSB_HD void rbCentralImpulse(Body& b, V3 imp) { b.lin = b.lin + (imp * V3{1, 1, 1}) * b.invMass; }
RSB_HD void rbTorqueImpulse(Body& b, V3 t) { b.ang = b.ang + (b.invIw * t) * V3{1, 1, 1}; }
RSB_HD void rbImpulse(Body& b, V3 imp, V3 relPos) {
    if (b.invMass != 0.f) {
        rbCentralImpulse(b, imp);
        rbTorqueImpulse(b, cross(relPos, imp * V3{1, 1, 1}));
    }
}
RSB_HD void rbCentralForce(Body& b, V3 f) { b.force = b.force + f * V3{1, 1, 1}; }
RSB_HD void rbTorque(Body& b, V3 t) { b.torque = b.torque + t * V3{1, 1, 1}; }
RSB_HD V3 rbVelAt(const Body& b, V3 rel) { return b.lin + cross(b.ang, rel); }
// btRigidBody::computeImpulseDenominator
RSB_HD float rbImpulseDenom(const Body& b, V3 pos, V3 normal) {
    V3 r0 = pos - b.xf.o;
    V3 c0 = cross(r0, normal);
    V3 vec = cross(tmul(c0, b.invIw), r0);
    return b.invMass + dot(normal, vec);
}

// Ground object seen by a wheel ray: a static shape or a dynamic body
struct GroundRef {
    V3 com;
    V3 lin, ang;
    M3 basis;
    V3 invInertiaLocal;
    float invMass;
    const Body* body;
};
RSB_HD GroundRef groundRef(const World& W, int o) {
    GroundRef g;
    if (o < OBJ_BALL) {
        g.com = o < MAX_MESHES ? v3zero() : W.S->planeOrigin[o - MAX_MESHES];
        g.lin = g.ang = v3zero();
        g.basis = m3identity();
        g.invInertiaLocal = v3zero();
        g.invMass = 0.f;
        g.body = nullptr;
    } else {
        const Body& b = W.b[o - OBJ_BALL];
        g.com = b.xf.o;
        g.lin = b.lin;
        g.ang = b.ang;
        g.basis = b.xf.b;
        g.invInertiaLocal = b.invIl;
        g.invMass = b.invMass;
        g.body = &b;
    }
    return g;
}

// resolveSingleBilateral (btContactConstraint.cpp:108-150)
RSB_HD float resolveBilateral(const Body& b1, V3 pos1, const GroundRef& g, V3 pos2, V3 normal) {
    float nl2 = length2(normal);
    if (nl2 > 1.1f) return 0.f;
    V3 rel1 = pos1 - b1.xf.o;
    V3 rel2 = pos2 - g.com;
    V3 vel1 = rbVelAt(b1, rel1);
    V3 vel2 = g.lin + cross(g.ang, rel2);
    V3 vel = vel1 - vel2;
    // btJacobianEntry (btJacobianEntry.h:35-53)
    V3 aJ = transpose(b1.xf.b) * cross(rel1, normal);
    V3 bJ = transpose(g.basis) * cross(rel2, -normal);
    V3 m0 = b1.invIl * aJ;
    V3 m1 = g.invInertiaLocal * bJ;
    float adiag = ((b1.invMass + dot(m0, aJ)) + g.invMass) + dot(m1, bJ);
    float jacInv = 1.f / adiag;
    float relVel = dot(normal, vel);
    return (-0.2f * relVel) * jacInv;
}

// resolveSingleCollision (btContactConstraint.cpp:60-105), impulses not applied
RSB_HD float resolveCollision(const Body& b1, int obj, const World& W, V3 contact, V3 normal, float distance, float timeStep) {
    GroundRef g = groundRef(W, obj);
    V3 rel1 = contact - b1.xf.o;
    V3 rel2 = contact - g.com;
    V3 vel1 = rbVelAt(b1, rel1);
    V3 vel2 = g.lin + cross(g.ang, rel2);
    V3 vel = vel1 - vel2;
    float relVel = dot(normal, vel);
    float restitution = 0.f * -relVel;
    float positionalError = (0.2f * -distance) / timeStep;
    float velocityError = -(1.0f + restitution) * relVel;
    float denom0 = rbImpulseDenom(b1, contact, normal);
    float denom1 = 0.f;
    if (g.body) denom1 = rbImpulseDenom(*g.body, contact, normal);
    else {
        V3 r0 = contact - g.com;
        V3 c0 = cross(r0, normal);
        M3 zero = m3(0, 0, 0, 0, 0, 0, 0, 0, 0);
        denom1 = 0.f + dot(normal, cross(tmul(c0, zero), r0));
    }
    float jacInv = 1.f / (denom0 + denom1);
    float imp = positionalError * jacInv + velocityError * jacInv;
    return 0.f > imp ? 0.f : imp;
}

// ------------------------------------------------------------------ btVehicleRL

RSB_HD void wheelTransformsWS(const CarParams& C, const Body& cb, WheelTick& w, int i) {
    w.inContact = 0;
    w.withWorld = 0;
    w.hardPoint = xfPoint(cb.xf, C.wheelConn[i]);
    w.dirWS = cb.xf.b * V3{0, 0, -1};
    w.axleWS = cb.xf.b * V3{0, -1, 0};
}

// btVehicleRL::updateWheelTransform: basis of the steered wheel
RSB_HD void wheelTransform(const CarParams& C, const Body& cb, WheelTick& w, int i, float steerAngle) {
    wheelTransformsWS(C, cb, w, i);
    V3 up = -w.dirWS;
    V3 right = w.axleWS;
    V3 fwd = normalized(cross(up, right));
    M3 steer = m3fromQuat(qaxisAngle(up, steerAngle));
    // columns: forward (0) = fwd, right (1) = -right, up (2) = up
    M3 b2 = m3(fwd.x, -right.x, up.x, fwd.y, -right.y, up.y, fwd.z, -right.z, up.z);
    w.basis = steer * b2;
}

RSB_HD V3 chassisUp(const Body& cb) { return cb.xf.b.col(2); }
RSB_HD V3 chassisFwd(const Body& cb) { return cb.xf.b.col(0); }

// btVehicleRL::rayCast (btVehicleRL.cpp:118-206)
RSB_HD void wheelRayCast(World& W, int ci, int i) {
    const CarParams& C = W.P->car;
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    WheelTick& w = c.w[i];
    wheelTransformsWS(C, cb, w, i);
    float travel = C.susTravel;
    float rayLen = C.rayLen[i];
    V3 source = w.hardPoint;
    V3 target = source + w.dirWS * rayLen;
    w.contactPoint = target;
    w.ground = -1;
    V3 hp, hn;
    float frac;
    int obj = castRay(W, source, target, OBJ_CAR0 + ci, hp, hn, frac);
    if (obj >= 0) {
        w.contactPoint = hp;
        w.contactNormal = hn;
        w.inContact = 1;
        bool isStatic = obj < OBJ_BALL;
        w.withWorld = isStatic ? 1 : 0;
        w.ground = obj;
        V3 upv = chassisUp(cb);
        float traceLen = dot(w.hardPoint - w.contactPoint, upv);
        w.suspLen = traceLen - C.wheelRadius[i];
        float lo = C.susRest[i] - travel, hi = C.susRest[i] + travel;
        w.suspLen = (w.suspLen < lo) ? lo : ((hi < w.suspLen) ? hi : w.suspLen);
        float denom = dot(w.contactNormal, upv);
        V3 relpos = w.contactPoint - cb.xf.o;
        V3 velAt = rbVelAt(cb, relpos);
        float projVel = dot(w.contactNormal, velAt);
        if ((double)denom > 0.1) {
            float inv = 1.f / denom;
            w.relVel = projVel * inv;
            w.clippedInv = inv;
        } else {
            w.relVel = 0.f;
            w.clippedInv = 10.f;
        }
        if (isStatic) {
            float thresh = C.pushThresh[i];
            if (traceLen < thresh) {
                float delta = traceLen - thresh;
                float ts = W.tick == 0 ? (1.f / 60.f) : W.P->dt;  // btContactSolverInfo::m_timeStep
                float res = resolveCollision(cb, obj, W, hp, hn, delta, ts);
                c.extraPush[i] = res / 4.f;
            }
        }
    } else {
        w.suspLen = C.susRest[i] + travel;
        w.relVel = 0.f;
        w.contactNormal = -w.dirWS;
        w.clippedInv = 1.f;
        c.extraPush[i] = 0.f;
    }
}

// btVehicleRL::calcFrictionImpulses (btVehicleRL.cpp:307-370)
RSB_HD void calcFrictionImpulses(World& W, int ci, float timeStep) {
    const CarParams& C = W.P->car;
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    float frictionScale = C.mass / 3.f;
    for (int i = 0; i < 4; i++) {
        WheelTick& w = c.w[i];
        if (w.ground >= 0) {
            GroundRef g = groundRef(W, w.ground);
            V3 axle = w.basis.col(1);
            V3 surf = w.contactNormal;
            float proj = dot(axle, surf);
            axle = axle - surf * proj;
            axle = safeNormalized(axle);
            V3 fwd = safeNormalized(cross(surf, axle));
            float side = resolveBilateral(cb, w.contactPoint, g, w.contactPoint, axle);
            float rolling;
            float engineForce = c.engineForce, brake = c.brake;
            if (engineForce == 0.f) {
                if (brake != 0.f) {
                    V3 carRel = w.contactPoint - cb.xf.o;
                    V3 v1 = rbVelAt(cb, carRel);
                    V3 v2 = g.lin + cross(g.ang, carRel);
                    V3 cv = v1 - v2;
                    float relVel = dot(cv, fwd);
                    if (timeStep > (1 / 80.f)) {
                        float threshold = -(1 / (timeStep * 150.f)) + 0.8f;
                        if (fabsf(relVel) < threshold) relVel = 0;
                    }
                    float rf = -relVel * 113.73963f;
                    rolling = fmin_(fmax_(rf, -brake), brake);
                } else {
                    rolling = 0.f;
                }
            } else {
                rolling = -engineForce / frictionScale;
            }
            V3 total = ((fwd * rolling) * c.longF[i]) + ((axle * side) * c.latF[i]);
            w.impulse = total * frictionScale;
        } else {
            w.impulse = v3zero();
        }
    }
}

// btVehicleRL::updateSuspension (btVehicleRL.cpp:275-305)
RSB_HD void updateSuspension(World& W, int ci, float dt) {
    const CarParams& C = W.P->car;
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    for (int i = 0; i < 4; i++) {
        WheelTick& w = c.w[i];
        if (w.inContact) {
            float force = ((C.susRest[i] - w.suspLen) * SUSPENSION_STIFFNESS) * w.clippedInv;
            float damp = (w.relVel < 0) ? WHEELS_DAMPING_COMPRESSION : WHEELS_DAMPING_RELAXATION;
            w.susForce = force - (damp * w.relVel);
            w.susForce *= C.susForceScale[i];
            if (w.susForce < 0) w.susForce = 0;
        } else {
            w.susForce = 0;
        }
    }
    for (int i = 0; i < 4; i++) {
        WheelTick& w = c.w[i];
        if (w.susForce != 0) {
            V3 off = w.contactPoint - cb.xf.o;
            float base = (w.susForce * dt) + c.extraPush[i];
            V3 f = w.contactNormal * base;
            rbImpulse(cb, f, off);
        }
    }
}

// btVehicleRL::applyFrictionImpulses (btVehicleRL.cpp:372-387)
RSB_HD void applyFrictionImpulses(World& W, int ci, float dt) {
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    V3 up = chassisUp(cb);
    for (int i = 0; i < 4; i++) {
        WheelTick& w = c.w[i];
        if (!isZero(w.impulse)) {
            V3 off = w.contactPoint - cb.xf.o;
            float d = dot(up, off);
            V3 rel = off - up * d;
            rbImpulse(cb, w.impulse * dt, rel);
        }
    }
}

// btVehicleRL::getUpwardsDirFromWheelContacts
RSB_HD V3 upwardsDirFromWheels(const World& W, int ci) {
    const CarSim& c = W.c[ci];
    V3 sum = v3zero();
    for (int i = 0; i < 4; i++)
        if (c.w[i].inContact) sum = sum + c.w[i].contactNormal;
    if (sum == v3zero()) return chassisUp(W.b[1 + ci]);
    return safeNormalized(sum);
}

// ------------------------------------------------------------------ Car

RSB_HD float clampf(float v, float lo, float hi) {
    float m = (v > lo) ? v : lo;
    return (m < hi) ? m : hi;
}
RSB_HD int sgnf(float v) { return (v > 0) - (v < 0); }

RSB_HD bool cflag(const CarSim& c, uint32_t f) { return (c.flags & f) != 0; }
RSB_HD void setFlag(CarSim& c, uint32_t f, bool on) { c.flags = on ? (c.flags | f) : (c.flags & ~f); }

// Car::SetState applied to a fresh CarState with the given placement (Car.cpp:24-36)
RSB_HD void carSetSpawnState(World& W, int ci, V3 posUu, const M3& rot, float boost) {
    CarSim& c = W.c[ci];
    Body& b = W.b[1 + ci];
    b.xf.o = posUu * kUuToBt;
    b.xf.b = rot;
    b.lin = V3{0, 0, 0} * kUuToBt;
    b.ang = v3zero();
    b.invIw = scaled(b.xf.b, b.invIl) * transpose(b.xf.b);
    c.velCache = v3zero();
    uint32_t keepTeam = c.flags & CF_TEAM_ORANGE;
    c.flags = CF_ON_GROUND | keepTeam;
    c.boost = boost;
    c.timeSpentBoosting = c.jumpTime = c.flipTime = c.airTime = c.airTimeSinceJump = 0.f;
    c.supersonicTime = c.handbrakeVal = c.autoFlipTimer = c.autoFlipTorqueScale = 0.f;
    c.demoRespawnTimer = c.carContactCooldown = 0.f;
    c.flipRelTorque = c.worldContactNormal = v3zero();
    c.carContactOtherId = 0;
    c.ballHitTick = c.ballHitExtraTick = ~0ull;
    c.ballHitRelPos = c.ballHitBallPos = c.ballHitExtraVel = v3zero();
    c.rotMat = rot;
    for (int k = 0; k < 5; k++) c.lastCtl[k] = 0.f;
    c.lastCtlBits = 0;
}

// Car::Respawn for soccar; `pick` selects one of CAR_RESPAWN_LOCATIONS_SOCCAR
RSB_HD void carRespawn(World& W, int ci, int pick) {
    W.cull &= ~(1u << (1 + ci));  // the spawn is next to the floor: no culling this launch
    const double kRespawnYaw = 3.14159265358979323846 / 2;
    const float xs[4] = {-2304.f, -2688.f, 2304.f, 2688.f};
    CarSim& c = W.c[ci];
    bool blue = c.team == 0;
    float y = -4608.f * (blue ? 1.f : -1.f);
    V3 pos{xs[pick], y, CAR_RESPAWN_Z};
    float yaw = (float)(kRespawnYaw + (blue ? 0.0 : 3.14159265358979323846));
    // Angle(yaw, 0, 0).ToRotMat() = setEulerYPR(yaw, -0, -0) = setEulerZYX(-0, -0, yaw)
    M3 rot = m3fromEulerZYX(-0.f, -0.f, yaw);
    carSetSpawnState(W, ci, pos, rot, W.P->car.spawnBoost);
}

// Car::_UpdateWheels (Car.cpp:323-461)
RSB_HD void updateWheels(World& W, int ci, float dt, int numContact, float fwdSpeedUu) {
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    float absFwd = fabsf(fwdSpeedUu);
    bool worldContact = false;
    for (int i = 0; i < 4; i++) worldContact |= c.w[i].withWorld != 0;
    bool handbrake = (c.ctlBits & 4u) != 0, boostIn = (c.ctlBits & 2u) != 0;
    if (handbrake) c.handbrakeVal += POWERSLIDE_RISE_RATE * dt;
    else c.handbrakeVal -= POWERSLIDE_FALL_RATE * dt;
    c.handbrakeVal = clampf(c.handbrakeVal, 0, 1);
    float realThrottle = c.ctl[0];
    float realBrake = 0;
    if (boostIn && c.boost > 0) realThrottle = 1;
    {
        float driveSpeedScale = curveOut(crvDriveTorque(), absFwd);
        float engineThrottle = realThrottle;
        if (!handbrake) {
            float absThrottle = fabsf(realThrottle);
            if (absThrottle >= THROTTLE_DEADZONE) {
                if (absFwd > STOPPING_FORWARD_VEL && sgnf(realThrottle) != sgnf(fwdSpeedUu)) {
                    realBrake = 1;
                    if (absFwd > BRAKING_NO_THROTTLE_SPEED_THRESH) engineThrottle = 0;
                }
            } else {
                engineThrottle = 0;
                bool fullStop = (absFwd < STOPPING_FORWARD_VEL);
                realBrake = fullStop ? 1 : COASTING_BRAKE_FACTOR;
            }
        }
        if (numContact < 3) driveSpeedScale /= 4;
        float engine = (engineThrottle * (THROTTLE_TORQUE_AMOUNT * kUuToBt)) * driveSpeedScale;
        float brakeF = realBrake * (BRAKE_TORQUE_AMOUNT * kUuToBt);
        c.engineForce = engine;
        c.brake = brakeF;
    }
    {
        float steerAngle = curveOut(crvSteerAngle(), absFwd);
        if (c.handbrakeVal != 0.f)
            steerAngle += (curveOut(crvPowerslideSteer(), absFwd) - steerAngle) * c.handbrakeVal;
        steerAngle *= c.ctl[1];
        c.steerAngle = steerAngle;
    }
    for (int i = 0; i < 4; i++) {
        WheelTick& w = c.w[i];
        if (w.ground >= 0) {
            V3 vel = cb.lin, angVel = cb.ang;
            V3 latDir = w.basis.col(1);
            V3 longDir = cross(latDir, w.contactNormal);
            float fci = 0;
            V3 wheelDelta = w.hardPoint - cb.xf.o;
            V3 crossVec = (cross(angVel, wheelDelta) + vel) * kBtToUu;
            float baseFriction = fabsf(dot(crossVec, latDir));
            if (baseFriction > 5) fci = baseFriction / (fabsf(dot(crossVec, longDir)) + baseFriction);
            float lat = curveOut(crvLatFriction(), fci);
            float lon = curveOut(crvLongFriction(), fci);
            if (c.handbrakeVal != 0.f) {
                float hb = c.handbrakeVal;
                lat *= (curveOut(crvHandbrakeLat(), fci) - 1) * hb + 1;
                lon *= (curveOut(crvHandbrakeLong(), fci) - 1) * hb + 1;
            } else {
                lon = 1;
            }
            bool sticky = realThrottle != 0;
            if (!sticky) {
                float ns = curveOut(crvNonSticky(), w.contactNormal.z);
                lat *= ns;
                lon *= ns;
            }
            c.latF[i] = lat;
            c.longF[i] = lon;
        }
    }
    if (worldContact) {
        V3 up = upwardsDirFromWheels(W, ci);
        bool fullStick = (realThrottle != 0) || (absFwd > STOPPING_FORWARD_VEL);
        float scale = 0.5f;
        if (fullStick) scale += 1 - fabsf(up.z);
        rbCentralForce(cb, ((up * scale) * (GRAVITY_Z * kUuToBt)) * CAR_MASS_BT);
    }
}

// Car::_UpdateAirTorque (Car.cpp:558-646)
RSB_HD void updateAirTorque(World& W, int ci, bool updateAirControl) {
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    V3 dirPitch = -c.rotMat.col(1), dirYaw = c.rotMat.col(2), dirRoll = -c.rotMat.col(0);
    float pitch = c.ctl[2], yaw = c.ctl[3], roll = c.ctl[4];
    bool doAir = false;
    if (cflag(c, CF_IS_FLIPPING)) setFlag(c, CF_IS_FLIPPING, cflag(c, CF_HAS_FLIPPED) && c.flipTime < FLIP_TORQUE_TIME);
    if (cflag(c, CF_IS_FLIPPING)) {
        V3 rel = c.flipRelTorque;
        if (!isZero(c.flipRelTorque)) {
            float pitchScale = 1;
            if (rel.y != 0 && pitch != 0) {
                if (sgnf(rel.y) == sgnf(pitch)) {
                    pitchScale = 1 - fmin_(fabsf(pitch), 1);
                    doAir = true;
                }
            }
            rel.y *= pitchScale;
            V3 dodgeTorque = rel * V3{FLIP_TORQUE_X, FLIP_TORQUE_Y, 0};
            rbTorque(cb, (inverse(cb.invIw) * cb.xf.b) * dodgeTorque);
        } else {
            doAir = true;
        }
    } else {
        doAir = true;
    }
    doAir = doAir && !cflag(c, CF_AUTO_FLIPPING);
    doAir = doAir && updateAirControl;
    if (doAir) {
        float pitchTorqueScale = 1;
        V3 torque;
        if (pitch != 0 || yaw != 0 || roll != 0) {
            if (cflag(c, CF_IS_FLIPPING)) pitchTorqueScale = 0;
            else if (cflag(c, CF_HAS_FLIPPED)) {
                if (c.flipTime < FLIP_TORQUE_TIME + FLIP_PITCHLOCK_EXTRA_TIME) pitchTorqueScale = 0;
            }
            torque = (((dirPitch * pitch) * pitchTorqueScale) * CAR_AIR_CONTROL_TORQUE_X) +
                     ((dirYaw * yaw) * CAR_AIR_CONTROL_TORQUE_Y) + ((dirRoll * roll) * CAR_AIR_CONTROL_TORQUE_Z);
        } else {
            torque = v3zero();
        }
        V3 angVel = cb.ang;
        float dampPitch = (dot(dirPitch, angVel) * CAR_AIR_CONTROL_DAMPING_X) * (1 - fabsf(doAir ? (pitch * pitchTorqueScale) : 0));
        float dampYaw = (dot(dirYaw, angVel) * CAR_AIR_CONTROL_DAMPING_Y) * (1 - fabsf(doAir ? yaw : 0));
        float dampRoll = dot(dirRoll, angVel) * CAR_AIR_CONTROL_DAMPING_Z;
        V3 damping = ((dirYaw * dampYaw) + (dirPitch * dampPitch)) + (dirRoll * dampRoll);
        rbTorque(cb, (inverse(cb.invIw) * (torque - damping)) * CAR_TORQUE_SCALE);
    }
    float throttle = c.ctl[0];
    if (throttle != 0)
        rbCentralForce(cb, (((c.rotMat.col(0) * throttle) * THROTTLE_AIR_ACCEL) * kUuToBt) * CAR_MASS_BT);
}

// Car::_UpdateJump (Car.cpp:496-556)
RSB_HD void updateJump(World& W, int ci, float dt, bool jumpPressed) {
    const CarParams& C = W.P->car;
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    bool jump = (c.ctlBits & 1u) != 0;
    if (cflag(c, CF_ON_GROUND) && !cflag(c, CF_IS_JUMPING)) {
        if (cflag(c, CF_HAS_JUMPED) && c.jumpTime < JUMP_MIN_TIME + JUMP_RESET_TIME_PAD) {
        } else {
            setFlag(c, CF_HAS_JUMPED, false);
            c.jumpTime = 0;
        }
    }
    if (cflag(c, CF_IS_JUMPING)) {
        setFlag(c, CF_IS_JUMPING, c.jumpTime < JUMP_MIN_TIME || (jump && c.jumpTime < JUMP_MAX_TIME));
    } else if (cflag(c, CF_ON_GROUND) && jumpPressed) {
        setFlag(c, CF_IS_JUMPING, true);
        c.jumpTime = 0;
        V3 f = ((c.rotMat.col(2) * C.jumpImmediateForce) * kUuToBt) * CAR_MASS_BT;
        rbCentralImpulse(cb, f);
    }
    if (cflag(c, CF_IS_JUMPING)) {
        setFlag(c, CF_HAS_JUMPED, true);
        V3 total = c.rotMat.col(2) * C.jumpAccel;
        if (c.jumpTime < JUMP_MIN_TIME) total *= 0.62f;
        rbCentralForce(cb, (total * kUuToBt) * CAR_MASS_BT);
    }
    if (cflag(c, CF_IS_JUMPING) || cflag(c, CF_HAS_JUMPED)) c.jumpTime += dt;
}

// Car::_UpdateAutoFlip (Car.cpp:770-803)
RSB_HD void updateAutoFlip(World& W, int ci, float dt, bool jumpPressed) {
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    if (jumpPressed && cflag(c, CF_WORLD_CONTACT) && c.worldContactNormal.z > CAR_AUTOFLIP_NORMZ_THRESH) {
        // Angle::FromRotMat -> btMatrix3x3::getEulerYPR; roll is negated
        const M3& m = c.rotMat;
        float rollB = rsAtan2f(m.r[2].y, m.r[2].z);
        float sp = -m.r[2].x;
        sp = sp < -1.f ? -1.f : (sp > 1.f ? 1.f : sp);
        float pitchB = rsAsinf(sp);
        if (fabsf(pitchB) == kHalfPi) {
            if (rollB > 0) rollB -= kPi;
            else rollB += kPi;
        }
        float roll = rollB * -1;
        float absRoll = fabsf(roll);
        if (absRoll > CAR_AUTOFLIP_ROLL_THRESH) {
            c.autoFlipTimer = (float)((double)CAR_AUTOFLIP_TIME * ((double)absRoll / 3.14159265358979323846));
            c.autoFlipTorqueScale = (roll > 0) ? 1.f : -1.f;
            setFlag(c, CF_AUTO_FLIPPING, true);
            rbCentralImpulse(cb, ((-c.rotMat.col(2) * CAR_AUTOFLIP_IMPULSE) * kUuToBt) * CAR_MASS_BT);
        }
    }
    if (cflag(c, CF_AUTO_FLIPPING)) {
        if (c.autoFlipTimer <= 0) {
            setFlag(c, CF_AUTO_FLIPPING, false);
            c.autoFlipTimer = 0;
        } else {
            cb.ang = cb.ang + ((c.rotMat.col(0) * CAR_AUTOFLIP_TORQUE) * c.autoFlipTorqueScale) * dt;
            c.autoFlipTimer -= dt;
        }
    }
}

// Car::_UpdateDoubleJumpOrFlip (Car.cpp:648-768)
RSB_HD void updateDoubleJumpOrFlip(World& W, int ci, float dt, bool jumpPressed, float fwdSpeedUu) {
    const CarParams& C = W.P->car;
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    float pitch = c.ctl[2], yaw = c.ctl[3], roll = c.ctl[4];
    if (cflag(c, CF_ON_GROUND)) {
        setFlag(c, CF_HAS_DOUBLE_JUMPED, false);
        setFlag(c, CF_HAS_FLIPPED, false);
        c.airTime = 0;
        c.airTimeSinceJump = 0;
        c.flipTime = 0;
    } else {
        c.airTime += dt;
        if (cflag(c, CF_HAS_JUMPED) && !cflag(c, CF_IS_JUMPING)) c.airTimeSinceJump += dt;
        else c.airTimeSinceJump = 0;
        if (jumpPressed && c.airTimeSinceJump < DOUBLEJUMP_MAX_DELAY) {
            float inputMag = (fabsf(yaw) + fabsf(pitch)) + fabsf(roll);
            bool isFlipInput = inputMag >= C.dodgeDeadzone;
            bool fresh = !cflag(c, CF_HAS_DOUBLE_JUMPED) && !cflag(c, CF_HAS_FLIPPED);
            bool canUse = isFlipInput ? (fresh || C.unlimitedFlips) : (fresh || C.unlimitedDoubleJumps);
            if (cflag(c, CF_AUTO_FLIPPING)) canUse = false;
            if (canUse) {
                if (isFlipInput) {
                    c.flipTime = 0;
                    setFlag(c, CF_HAS_FLIPPED, true);
                    setFlag(c, CF_IS_FLIPPING, true);
                    float fwdRatio = fabsf(fwdSpeedUu) / CAR_MAX_SPEED;
                    V3 dodgeDir = V3{-pitch, yaw + roll, 0};
                    if (fabsf(yaw + roll) < 0.1f && fabsf(pitch) < 0.1f) dodgeDir = v3zero();
                    else dodgeDir = safeNormalized(dodgeDir);
                    c.flipRelTorque = V3{-dodgeDir.y, dodgeDir.x, 0};
                    if (fabsf(dodgeDir.x) < 0.1f) dodgeDir.x = 0;
                    if (fabsf(dodgeDir.y) < 0.1f) dodgeDir.y = 0;
                    if (!fuzzyZero(dodgeDir)) {
                        bool back;
                        if (fabsf(fwdSpeedUu) < 100.0f) back = dodgeDir.x < 0.0f;
                        else back = (dodgeDir.x >= 0.0f) != (fwdSpeedUu >= 0.0f);
                        V3 iv = dodgeDir * FLIP_INITIAL_VEL_SCALE;
                        float maxX = back ? FLIP_BACKWARD_IMPULSE_MAX_SPEED_SCALE : FLIP_FORWARD_IMPULSE_MAX_SPEED_SCALE;
                        iv.x *= ((maxX - 1) * fwdRatio) + 1.f;
                        iv.y *= ((FLIP_SIDE_IMPULSE_MAX_SPEED_SCALE - 1) * fwdRatio) + 1.f;
                        if (back) iv.x *= FLIP_BACKWARD_IMPULSE_SCALE_X;
                        V3 fd = c.rotMat.col(0);
                        float ang = rsAtan2f(fd.y, fd.x);
                        V3 xDir{rsCosf(ang), -rsSinf(ang), 0.f}, yDir{rsSinf(ang), rsCosf(ang), 0.f};
                        V3 dv{dot(iv, xDir), dot(iv, yDir), 0.f};
                        rbCentralImpulse(cb, (dv * kUuToBt) * CAR_MASS_BT);
                    }
                } else {
                    rbCentralImpulse(cb, ((c.rotMat.col(2) * JUMP_IMMEDIATE_FORCE) * kUuToBt) * CAR_MASS_BT);
                    setFlag(c, CF_HAS_DOUBLE_JUMPED, true);
                }
            }
        }
    }
    if (cflag(c, CF_IS_FLIPPING)) {
        c.flipTime += dt;
        if (c.flipTime <= FLIP_TORQUE_TIME) {
            if (c.flipTime >= FLIP_Z_DAMP_START && (cb.lin.z < 0 || c.flipTime < FLIP_Z_DAMP_END)) cb.lin.z *= C.flipZDamp;
        }
    } else if (cflag(c, CF_HAS_FLIPPED)) {
        c.flipTime += dt;
    }
}

// Car::_UpdateAutoRoll (Car.cpp:805-832)
RSB_HD void updateAutoRoll(World& W, int ci, int numContact) {
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    V3 groundUp = numContact > 0 ? upwardsDirFromWheels(W, ci) : c.worldContactNormal;
    V3 groundDown = -groundUp;
    V3 fwd = c.rotMat.col(0), right = c.rotMat.col(1);
    V3 crossRight = cross(groundUp, fwd);
    V3 crossFwd = cross(groundDown, crossRight);
    float rightF = 1 - clampf(dot(right, crossRight), 0, 1);
    float fwdF = 1 - clampf(dot(fwd, crossFwd), 0, 1);
    V3 tdRight = fwd * (dot(right, groundUp) >= 0 ? -1.f : 1.f);
    V3 tdFwd = right * (dot(fwd, groundUp) >= 0 ? 1.f : -1.f);
    V3 tRight = tdRight * rightF;
    V3 tFwd = tdFwd * fwdF;
    rbCentralForce(cb, ((groundDown * CAR_AUTOROLL_FORCE) * kUuToBt) * CAR_MASS_BT);
    rbTorque(cb, (inverse(cb.invIw) * (tFwd + tRight)) * CAR_AUTOROLL_TORQUE);
}

// Car::_UpdateBoost (Car.cpp:463-494)
RSB_HD void updateBoost(World& W, int ci, float dt) {
    const CarParams& C = W.P->car;
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    bool boostIn = (c.ctlBits & 2u) != 0;
    if (c.timeSpentBoosting > 0) {
        if (!boostIn && c.timeSpentBoosting >= BOOST_MIN_TIME) c.timeSpentBoosting = 0;
        else c.timeSpentBoosting += dt;
    } else {
        if (boostIn) c.timeSpentBoosting = dt;
    }
    if (c.boost > 0 && c.timeSpentBoosting > 0) {
        c.boost = fmax_(c.boost - C.boostUsedPerSecond * dt, 0);
        float accel = cflag(c, CF_ON_GROUND) ? C.boostAccelGround : C.boostAccelAir;
        rbCentralForce(cb, (c.rotMat.col(0) * (accel * kUuToBt)) * CAR_MASS_BT);
    }
    c.boost = fmin_(c.boost, BOOST_MAX);
}

// Car::_PreTickUpdate
RSB_HD void carPreTick(World& W, int ci, uint32_t respawnPick) {
    const float dt = W.P->dt;
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    for (int k = 0; k < 5; k++) c.ctl[k] = clampf(c.ctl[k], -1, 1);
    if (cflag(c, CF_DEMOED)) {
        c.demoRespawnTimer = fmax_(c.demoRespawnTimer - dt, 0);
        if (c.demoRespawnTimer == 0) carRespawn(W, ci, (int)(respawnPick & 3u));
        cb.act = ACT_DISABLE_SIM;
        cb.noResp = 1;
    } else {
        cb.act = ACT_ACTIVE;
        cb.noResp = 0;
    }
    if (cflag(c, CF_DEMOED)) return;

    // btVehicleRL::updateVehicleFirst
    for (int i = 0; i < 4; i++) wheelTransform(W.P->car, cb, c.w[i], i, i < 2 ? c.steerAngle : 0.f);
    for (int i = 0; i < 4; i++) wheelRayCast(W, ci, i);
    calcFrictionImpulses(W, ci, dt);

    bool jump = (c.ctlBits & 1u) != 0, lastJump = (c.lastCtlBits & 1u) != 0;
    bool jumpPressed = jump && !lastJump;
    int numContact = 0;
    c.flags &= ~(0xFu * CF_WHEEL0);
    for (int i = 0; i < 4; i++) {
        if (c.w[i].inContact) c.flags |= CF_WHEEL0 << i;
        numContact += c.w[i].inContact ? 1 : 0;
    }
    setFlag(c, CF_ON_GROUND, numContact >= 3);
    float fwdSpeedUu = dot(cb.lin, chassisFwd(cb)) * kBtToUu;
    updateWheels(W, ci, dt, numContact, fwdSpeedUu);
    if (numContact < 3) updateAirTorque(W, ci, numContact == 0);
    else setFlag(c, CF_IS_FLIPPING, false);
    updateJump(W, ci, dt, jumpPressed);
    updateAutoFlip(W, ci, dt, jumpPressed);
    updateDoubleJumpOrFlip(W, ci, dt, jumpPressed, fwdSpeedUu);
    if (c.ctl[0] != 0 && ((numContact > 0 && numContact < 4) || cflag(c, CF_WORLD_CONTACT))) updateAutoRoll(W, ci, numContact);
    setFlag(c, CF_WORLD_CONTACT, false);
    // btVehicleRL::updateVehicleSecond
    updateSuspension(W, ci, dt);
    applyFrictionImpulses(W, ci, dt);
    updateBoost(W, ci, dt);
}

// Car::_PostTickUpdate + Car::_FinishPhysicsTick
RSB_HD void carPostTick(World& W, int ci) {
    const float dt = W.P->dt;
    Body& cb = W.b[1 + ci];
    CarSim& c = W.c[ci];
    if (cflag(c, CF_DEMOED)) return;
    c.rotMat = cb.xf.b;
    {
        float sp2 = length2(cb.lin * kBtToUu);
        bool ss;
        if (cflag(c, CF_SUPERSONIC) && c.supersonicTime < SUPERSONIC_MAINTAIN_MAX_TIME)
            ss = sp2 >= SUPERSONIC_MAINTAIN_MIN_SPEED * SUPERSONIC_MAINTAIN_MIN_SPEED;
        else
            ss = sp2 >= SUPERSONIC_START_SPEED * SUPERSONIC_START_SPEED;
        setFlag(c, CF_SUPERSONIC, ss);
        if (ss) c.supersonicTime += dt;
        else c.supersonicTime = 0;
    }
    if (c.carContactCooldown > 0) c.carContactCooldown = fmax_(c.carContactCooldown - dt, 0);
    for (int k = 0; k < 5; k++) c.lastCtl[k] = c.ctl[k];
    c.lastCtlBits = c.ctlBits;
    // _FinishPhysicsTick
    if (!isZero(c.velCache)) {
        cb.lin = cb.lin + c.velCache;
        c.velCache = v3zero();
    }
    V3 vel = cb.lin, ang = cb.ang;
    const float maxV = CAR_MAX_SPEED * kUuToBt;
    if (length2(vel) > maxV * maxV) vel = normalized(vel) * maxV;
    if (length2(ang) > CAR_MAX_ANG_SPEED * CAR_MAX_ANG_SPEED) ang = normalized(ang) * CAR_MAX_ANG_SPEED;
    cb.lin = vel;
    cb.ang = ang;
}

}  // namespace rsb
