// ABC front end of the B200 `rw; st` path: registers the GPU commands of
// CULS's ABC patch (src/abc_patch/abc_patch.cpp:31-54,
// abc_patch_gpucmd.cpp:237-251) -- gget, gput, grw, gst, gb, gps -- in an ABC
// binary, over the C ABI of libculs_b200.so.  The conversion and the command
// state are in abc_bridge.hpp (tested without ABC); this file only reads and
// builds ABC networks and hooks the commands in.
//
// Needs an ABC source tree (its headers and objects); built by
// build_abc_patch.sh only when CULS_ABC_ROOT names one.  No ABC tree exists
// on the machines this repository is built and tested on, so this file is
// compiled nowhere here.
extern "C" {
#include "base/abc/abc.h"
#include "base/main/main.h"
#include "base/main/mainInt.h"
#include "misc/extra/extra.h"
}

#include "abc_bridge.hpp"

namespace {

culs_abc::Session *g_session = nullptr;

// Abc_Obj_t pointers may carry ABC's complement bit; the builder keeps the
// regular node and reports the bit.
struct AbcBuilder {
    using Handle = Abc_Obj_t *;
    Abc_Ntk_t *ntk;
    Handle const1() { return Abc_AigConst1(ntk); }
    Handle pi() { return Abc_NtkCreatePi(ntk); }
    Handle po() { return Abc_NtkCreatePo(ntk); }
    Handle and2(Handle x, bool cx, Handle y, bool cy, bool *c) {
        Abc_Obj_t *r = Abc_AigAnd((Abc_Aig_t *)ntk->pManFunc, Abc_ObjNotCond(x, cx), Abc_ObjNotCond(y, cy));
        *c = Abc_ObjIsComplement(r) != 0;
        return Abc_ObjRegular(r);
    }
    void drive(Handle po, Handle d, bool c) { Abc_ObjAddFanin(po, Abc_ObjNotCond(d, c)); }
};

// gget: a strashed network's view (inputs, DFS-ordered AND nodes, outputs)
int CmdGet(Abc_Frame_t *pAbc, int argc, char **argv) {
    (void)argc;
    (void)argv;
    Abc_Ntk_t *ntk = Abc_FrameReadNtk(pAbc);
    if (!ntk || !Abc_NtkIsStrash(ntk)) {
        Abc_Print(-1, "gget: strash the network first.\n");
        return 1;
    }
    culs_abc::NtkView v;
    v.const1 = Abc_ObjId(Abc_AigConst1(ntk));
    for (int i = 0; i < Abc_NtkCiNum(ntk); i++) v.ci.push_back(Abc_ObjId(Abc_NtkCi(ntk, i)));
    Vec_Ptr_t *nodes = Abc_NtkDfs(ntk, 0);
    for (int i = 0; i < Vec_PtrSize(nodes); i++) {
        Abc_Obj_t *n = (Abc_Obj_t *)Vec_PtrEntry(nodes, i);
        v.ands.push_back({(int)Abc_ObjId(n), (int)Abc_ObjId(Abc_ObjFanin0(n)), Abc_ObjFaninC0(n),
                          (int)Abc_ObjId(Abc_ObjFanin1(n)), Abc_ObjFaninC1(n)});
    }
    Vec_PtrFree(nodes);
    for (int i = 0; i < Abc_NtkCoNum(ntk); i++) {
        Abc_Obj_t *co = Abc_NtkCo(ntk, i);
        v.co.push_back({(int)Abc_ObjId(Abc_ObjFanin0(co)), Abc_ObjFaninC0(co)});
    }
    return g_session->get(v);
}

// gput: the held graph back as a new strashed network
int CmdPut(Abc_Frame_t *pAbc, int argc, char **argv) {
    (void)argc;
    (void)argv;
    culs_abc::HostAig a;
    if (g_session->put(a)) return 1;
    Abc_Ntk_t *ntk = Abc_NtkAlloc(ABC_NTK_STRASH, ABC_FUNC_AIG, 1);
    Abc_Ntk_t *old = Abc_FrameReadNtk(pAbc);
    if (old && old->pName) ntk->pName = Extra_UtilStrsav(old->pName);
    if (old && old->pSpec) ntk->pSpec = Extra_UtilStrsav(old->pSpec);
    AbcBuilder b{ntk};
    std::string err;
    if (!culs_abc::aig_to_ntk(a, b, err)) {
        Abc_Print(-1, "gput: %s\n", err.c_str());
        Abc_NtkDelete(ntk);
        return 1;
    }
    Abc_NtkAddDummyPiNames(ntk);
    Abc_NtkAddDummyPoNames(ntk);
    if (!Abc_NtkCheck(ntk)) {
        Abc_Print(-1, "gput: the network failed ABC's check\n");
        Abc_NtkDelete(ntk);
        return 1;
    }
    Abc_FrameReplaceCurrentNetwork(pAbc, ntk);
    return 0;
}

// grw [-z] [-d], gst [-c], gb [-s], gps, grf, gresyn2
int CmdGpu(Abc_Frame_t *pAbc, int argc, char **argv) {
    (void)pAbc;
    return g_session->command(argc, argv);
}

void PatchInit(Abc_Frame_t *pAbc) {
    g_session = new culs_abc::Session();
    Cmd_CommandAdd(pAbc, "GPU", "gget", CmdGet, 0);
    Cmd_CommandAdd(pAbc, "GPU", "gput", CmdPut, 1);
    for (const char *name : {"grw", "gst", "gb", "gps", "grf", "gresyn2"}) Cmd_CommandAdd(pAbc, "GPU", name, CmdGpu, 0);
}

void PatchEnd(Abc_Frame_t *pAbc) {
    (void)pAbc;
    delete g_session;
    g_session = nullptr;
}

Abc_FrameInitializer_t g_init = {PatchInit, PatchEnd, nullptr, nullptr};

// ABC runs the registered initializers when it starts its frame
struct Register {
    Register() { Abc_FrameAddInitializer(&g_init); }
} g_register;

}  // namespace
