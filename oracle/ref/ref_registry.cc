// Registry of built-in reactions for the oracle build of the reference code.
// The reference generates this function with registerBuiltinReactions.pl
// (elec/registerBuiltinReactions.pl:32-63); the oracle needs only BetterTT06.
// Test infrastructure only.
#include "reactionFactory.hh"
REACTION_FACTORY(BetterTT06)(OBJECT* obj, const double dt, const int numPoints, const ThreadTeam& group);
void registerBuiltinReactions() { registerReactionFactory("BetterTT06", reactionFactoryForBetterTT06); }
